/*
 * Test infrastructure (oracle): restarted GMRES with the semantics the reference
 * gets from PETSc.
 *
 * The reference solves both GFD systems with KSPGMRES + PCJACOBI + KSPSetFromOptions
 * (solver.cpp:196-204 density, solver.cpp:267-276 potential).  PETSc 3.5.1 / 3.6.1
 * (Makefile:3, vneumann_makefile:3) is not vendored in the reference, so this file
 * restates the published PETSc 3.5 algorithm on one rank:
 *   - KSPSolve_GMRES: zero initial guess, outer restart loop, DIVERGED_ITS when the
 *     total iteration count reaches max_it;
 *   - KSPInitialResidual with left preconditioning: r = B (b - A x), B = diag(A)^-1
 *     (PCJACOBI; a zero diagonal entry is replaced by 1);
 *   - KSPGMRESCycle: classical Gram-Schmidt with refinement "never" (the default
 *     KSPGMRESClassicalGramSchmidtOrthogonalization), happy-breakdown tolerance
 *     1e-30, Givens rotations as in KSPGMRESUpdateHessenberg, solution built by
 *     back substitution (KSPGMRESBuildSoln);
 *   - KSPConvergedDefault on the preconditioned residual estimate:
 *     ttol = max(rtol * ||B b||, atol) fixed at the first test, converged when
 *     rnorm <= ttol, diverged when rnorm >= dtol * rnorm0.
 * Defaults (rtol 1e-5, atol 1e-50, dtol 1e5, max_it 10000, restart 30) are PETSc's;
 * the reference's run lines override them from the command line (Makefile:31).
 *
 * Never linked into the product library.
 */
#include "gmres_petsc.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* th > 1: the loop runs on th OpenMP threads (as PETSc runs it on MPI ranks); th <= 1:
   serially, in index order */
static double vdot(int n, const double *a, const double *b, int th) {
  double s = 0.0;
  if (th > 1) {
#pragma omp parallel for num_threads(th) reduction(+ : s) schedule(static)
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
  }
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

static void csr_matvec(int n, const int *rp, const int *ci, const double *v, const double *x,
                       double *y, int th) {
#pragma omp parallel for num_threads(th > 1 ? th : 1) if (th > 1) schedule(static)
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
    y[i] = s;
  }
}

void oracle_gmres_defaults(oracle_gmres_params *p) {
  p->restart = 30;
  p->rtol = 1e-5;
  p->atol = 1e-50;
  p->dtol = 1e5;
  p->max_it = 10000;
  p->its = 0;
  p->rnorm = 0.0;
  p->reason = 0;
  p->threads = 1;
}

/* KSPConvergedDefault */
static int converged_default(int n_its, double rnorm, const oracle_gmres_params *p, double *ttol,
                             double *rnorm0) {
  if (n_its == 0) {
    *ttol = fmax(p->rtol * rnorm, p->atol);
    *rnorm0 = rnorm;
  }
  if (rnorm != rnorm) return ORACLE_KSP_DIVERGED_NANORINF;
  if (rnorm <= *ttol) return rnorm < p->atol ? ORACLE_KSP_CONVERGED_ATOL : ORACLE_KSP_CONVERGED_RTOL;
  if (rnorm >= p->dtol * (*rnorm0)) return ORACLE_KSP_DIVERGED_DTOL;
  return 0;
}

int oracle_gmres_csr(int n, const int *rp, const int *ci, const double *val, const double *b,
                     double *x, oracle_gmres_params *p) {
  const int m = p->restart > 0 ? p->restart : 30;
  const double haptol = 1e-30;
  const int th = p->threads;
  double *dinv = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *V = (double *)malloc(sizeof(double) * (size_t)n * (m + 1) + 8);
  double *tmp = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double *HH = (double *)calloc((size_t)(m + 1) * m, sizeof(double)); /* HH(i,j) = HH[j*(m+1)+i] */
  double *cc = (double *)calloc((size_t)m, sizeof(double));
  double *ss = (double *)calloc((size_t)m, sizeof(double));
  double *grs = (double *)calloc((size_t)m + 1, sizeof(double));
  double *lhh = (double *)calloc((size_t)m + 1, sizeof(double));
  double *nrs = (double *)calloc((size_t)m + 1, sizeof(double));
  if (!dinv || !V || !tmp || !HH || !cc || !ss || !grs || !lhh || !nrs) {
    free(dinv); free(V); free(tmp); free(HH); free(cc); free(ss); free(grs); free(lhh); free(nrs);
    return -1;
  }
  /* PCSetUp_Jacobi */
  for (int i = 0; i < n; ++i) {
    double d = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) d = val[k];
    dinv[i] = d == 0.0 ? 1.0 : 1.0 / d;
  }
  for (int i = 0; i < n; ++i) x[i] = 0.0; /* guess_zero */

  double ttol = 0.0, rnorm0 = 0.0;
  int its = 0, reason = 0, itcount = 0, guess_zero = 1;
  double res = 0.0;
  while (!reason) {
    /* KSPInitialResidual (left PC) -> V(0) */
    double *v0 = V;
    if (guess_zero) {
      for (int i = 0; i < n; ++i) v0[i] = dinv[i] * b[i];
    } else {
      csr_matvec(n, rp, ci, val, x, tmp, th);
      for (int i = 0; i < n; ++i) v0[i] = dinv[i] * (b[i] - tmp[i]);
    }
    /* KSPGMRESCycle */
    double res_norm = sqrt(vdot(n, v0, v0, th));
    if (res_norm != 0.0) {
      double s = 1.0 / res_norm;
      for (int i = 0; i < n; ++i) v0[i] *= s;
    }
    res = res_norm;
    grs[0] = res_norm;
    if (res == 0.0) {
      reason = ORACLE_KSP_CONVERGED_ATOL;
      break;
    }
    reason = converged_default(its, res, p, &ttol, &rnorm0);
    int it = 0;
    while (!reason && it < m && its < p->max_it) {
      double *vk = V + (size_t)it * n;
      double *w = V + (size_t)(it + 1) * n;
      /* KSP_PCApplyBAorAB: w = B A v_it */
      csr_matvec(n, rp, ci, val, vk, tmp, th);
      for (int i = 0; i < n; ++i) w[i] = dinv[i] * tmp[i];
      /* classical Gram-Schmidt, refinement never */
      for (int j = 0; j <= it; ++j) lhh[j] = -vdot(n, w, V + (size_t)j * n, th);
      for (int j = 0; j <= it; ++j) {
        const double *vj = V + (size_t)j * n;
        double a = lhh[j];
#pragma omp parallel for num_threads(th > 1 ? th : 1) if (th > 1) schedule(static)
        for (int i = 0; i < n; ++i) w[i] += a * vj[i];
      }
      double *hcol = HH + (size_t)it * (m + 1);
      for (int j = 0; j <= it; ++j) hcol[j] = -lhh[j];
      double tt = sqrt(vdot(n, w, w, th));
      if (tt != 0.0) {
        double s = 1.0 / tt;
        for (int i = 0; i < n; ++i) w[i] *= s;
      }
      hcol[it + 1] = tt;
      double hapbnd = fabs(tt / grs[it]);
      if (hapbnd > haptol) hapbnd = haptol;
      int hapend = tt < hapbnd;
      /* KSPGMRESUpdateHessenberg */
      double *hh = hcol;
      for (int j = 1; j <= it; ++j) {
        double t0 = hh[j - 1];
        hh[j - 1] = cc[j - 1] * t0 + ss[j - 1] * hh[j];
        hh[j] = cc[j - 1] * hh[j] - ss[j - 1] * t0;
      }
      if (!hapend) {
        double t = sqrt(hh[it] * hh[it] + hh[it + 1] * hh[it + 1]);
        if (t == 0.0) {
          reason = ORACLE_KSP_DIVERGED_NULL;
        } else {
          cc[it] = hh[it] / t;
          ss[it] = hh[it + 1] / t;
          grs[it + 1] = -(ss[it] * grs[it]);
          grs[it] = cc[it] * grs[it];
          hh[it] = cc[it] * hh[it] + ss[it] * hh[it + 1];
          res = fabs(grs[it + 1]);
        }
      } else {
        res = 0.0;
      }
      ++it;
      ++its;
      if (reason) break;
      reason = converged_default(its, res, p, &ttol, &rnorm0);
      if (hapend) {
        if (!reason) reason = ORACLE_KSP_DIVERGED_BREAKDOWN;
        break;
      }
    }
    /* KSPGMRESBuildSoln(GRS, x, x, ksp, it - 1) */
    int last = it - 1;
    if (last >= 0) {
      double *Hl = HH + (size_t)last * (m + 1);
      nrs[last] = Hl[last] != 0.0 ? grs[last] / Hl[last] : 0.0;
      for (int ii = 1; ii <= last; ++ii) {
        int k = last - ii;
        double t = grs[k];
        for (int j = k + 1; j <= last; ++j) t -= HH[(size_t)j * (m + 1) + k] * nrs[j];
        double hkk = HH[(size_t)k * (m + 1) + k];
        nrs[k] = hkk != 0.0 ? t / hkk : 0.0;
      }
      for (int i = 0; i < n; ++i) tmp[i] = 0.0;
      for (int j = 0; j <= last; ++j) {
        const double *vj = V + (size_t)j * n;
        double a = nrs[j];
        for (int i = 0; i < n; ++i) tmp[i] += a * vj[i];
      }
      for (int i = 0; i < n; ++i) x[i] += tmp[i];
    }
    itcount += it;
    if (itcount >= p->max_it) {
      if (!reason) reason = ORACLE_KSP_DIVERGED_ITS;
      break;
    }
    guess_zero = 0;
  }
  p->its = its;
  p->rnorm = res;
  p->reason = reason;
  free(dinv); free(V); free(tmp); free(HH); free(cc); free(ss); free(grs); free(lhh); free(nrs);
  return 0;
}
