/*
 * Test infrastructure (oracle): CPU least-squares solver used by the oracle and by
 * the shim that lets the reference's solver.cpp build without LAPACK.
 *
 * The reference calls LAPACKE_dgels(LAPACK_ROW_MAJOR, 'N', m, n, nrhs, A, n, B, nrhs)
 * at solver.cpp:106 (nrhs = lm = 17, the GFD weight matrix) and solver.cpp:342
 * (nrhs = 1, differentiation).  LAPACK 3.5.0 (Makefile:5) is not vendored in the
 * reference, so this file restates its published algorithm for the m >= n,
 * trans = 'N' case:
 *   dgels  -> dgeqr2 (unblocked Householder QR; n = 9 is below LAPACK's block size)
 *          -> dorm2r (apply Q^T to B)
 *          -> dtrtrs (upper-triangular solve, info = k when R(k,k) == 0)
 * with dlarfg / dlarf / dnrm2 / dlapy2 written in the loop order of the reference
 * BLAS.  dgels' equilibration step (only taken when max|A| is below ~1e-292 or
 * above ~1e292) is omitted: GFD moment matrices are O(1) by construction
 * (offsets scaled by the cell length, solver.cpp:87-100).
 *
 * Never linked into the product library.
 */
#include "lsq_householder.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* reference BLAS dnrm2 (scaled sum of squares) */
static double ref_dnrm2(int n, const double *x) {
  if (n < 1) return 0.0;
  if (n == 1) return fabs(x[0]);
  double scale = 0.0, ssq = 1.0;
  for (int i = 0; i < n; ++i) {
    if (x[i] != 0.0) {
      double a = fabs(x[i]);
      if (scale < a) {
        double r = scale / a;
        ssq = 1.0 + ssq * r * r;
        scale = a;
      } else {
        double r = a / scale;
        ssq += r * r;
      }
    }
  }
  return scale * sqrt(ssq);
}

static double ref_dlapy2(double x, double y) {
  double xa = fabs(x), ya = fabs(y);
  double w = xa > ya ? xa : ya;
  double z = xa < ya ? xa : ya;
  if (z == 0.0) return w;
  double r = z / w;
  return w * sqrt(1.0 + r * r);
}

/* dlarfg: generate H = I - tau v v^T with H [alpha; x] = [beta; 0], v(0) = 1. */
static void ref_dlarfg(int n, double *alpha, double *x, double *tau) {
  if (n <= 1) { *tau = 0.0; return; }
  double xnorm = ref_dnrm2(n - 1, x);
  if (xnorm == 0.0) { *tau = 0.0; return; }
  double beta = -copysign(ref_dlapy2(*alpha, xnorm), *alpha);
  const double safmin = 2.2250738585072014e-308 / 1.1102230246251565e-16;
  int knt = 0;
  if (fabs(beta) < safmin) {
    const double rsafmn = 1.0 / safmin;
    do {
      ++knt;
      for (int i = 0; i < n - 1; ++i) x[i] *= rsafmn;
      beta *= rsafmn;
      *alpha *= rsafmn;
    } while (fabs(beta) < safmin && knt < 20);
    xnorm = ref_dnrm2(n - 1, x);
    beta = -copysign(ref_dlapy2(*alpha, xnorm), *alpha);
  }
  *tau = (beta - *alpha) / beta;
  double scal = 1.0 / (*alpha - beta);
  for (int i = 0; i < n - 1; ++i) x[i] *= scal;
  for (int j = 0; j < knt; ++j) beta *= safmin;
  *alpha = beta;
}

/* dlarf('L'): C(m x n, column-major, ldc) := (I - tau v v^T) C */
static void ref_dlarf_left(int m, int n, const double *v, double tau, double *C, int ldc,
                           double *work) {
  if (tau == 0.0) return;
  /* iladlr/iladlc: trim trailing zeros of v and trailing zero columns of C */
  int lastv = m;
  while (lastv > 0 && v[lastv - 1] == 0.0) --lastv;
  if (lastv == 0) return;
  int lastc = n;
  while (lastc > 0) {
    const double *col = C + (size_t)(lastc - 1) * ldc;
    int nz = 0;
    for (int i = 0; i < lastv; ++i)
      if (col[i] != 0.0) { nz = 1; break; }
    if (nz) break;
    --lastc;
  }
  /* dgemv('T'): work = C^T v */
  for (int j = 0; j < lastc; ++j) {
    const double *col = C + (size_t)j * ldc;
    double t = 0.0;
    for (int i = 0; i < lastv; ++i) t += col[i] * v[i];
    work[j] = t;
  }
  /* dger: C -= tau v work^T */
  for (int j = 0; j < lastc; ++j) {
    if (work[j] != 0.0) {
      double t = -tau * work[j];
      double *col = C + (size_t)j * ldc;
      for (int i = 0; i < lastv; ++i) col[i] += v[i] * t;
    }
  }
}

int oracle_dgels_rowmajor(int m, int n, int nrhs, double *A, int lda, double *B, int ldb) {
  if (m < n || n <= 0 || nrhs <= 0) return -1;
  double *a = (double *)malloc(sizeof(double) * (size_t)m * n);
  double *b = (double *)malloc(sizeof(double) * (size_t)m * nrhs);
  double *tau = (double *)malloc(sizeof(double) * (size_t)n);
  int wn = n > nrhs ? n : nrhs;
  double *work = (double *)malloc(sizeof(double) * (size_t)wn);
  /* row-major -> column-major (what LAPACKE does before calling dgels) */
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) a[(size_t)j * m + i] = A[(size_t)i * lda + j];
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < nrhs; ++j) b[(size_t)j * m + i] = B[(size_t)i * ldb + j];

  /* dgeqr2 */
  for (int i = 0; i < n; ++i) {
    double *aii = a + (size_t)i * m + i;
    ref_dlarfg(m - i, aii, aii + 1, &tau[i]);
    if (i < n - 1) {
      double keep = *aii;
      *aii = 1.0;
      ref_dlarf_left(m - i, n - i - 1, aii, tau[i], a + (size_t)(i + 1) * m + i, m, work);
      *aii = keep;
    }
  }
  /* dorm2r('L','T'): B := Q^T B */
  for (int i = 0; i < n; ++i) {
    double *aii = a + (size_t)i * m + i;
    double keep = *aii;
    *aii = 1.0;
    ref_dlarf_left(m - i, nrhs, aii, tau[i], b + i, m, work);
    *aii = keep;
  }
  /* dtrtrs: singularity check then dtrsm('L','U','N','N') */
  int info = 0;
  for (int i = 0; i < n; ++i)
    if (a[(size_t)i * m + i] == 0.0) { info = i + 1; break; }
  if (info == 0) {
    for (int j = 0; j < nrhs; ++j) {
      double *bj = b + (size_t)j * m;
      for (int k = n - 1; k >= 0; --k) {
        if (bj[k] != 0.0) {
          bj[k] /= a[(size_t)k * m + k];
          for (int i = 0; i < k; ++i) bj[i] -= bj[k] * a[(size_t)k * m + i];
        }
      }
    }
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < nrhs; ++j) B[(size_t)i * ldb + j] = b[(size_t)j * m + i];
  }
  /* A is overwritten by its QR factor in LAPACK; callers here never reuse it */
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) A[(size_t)i * lda + j] = a[(size_t)j * m + i];
  free(a); free(b); free(tau); free(work);
  return info;
}
