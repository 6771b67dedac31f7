/*
 * Test infrastructure (oracle): single-rank implementation of the PETSc calls listed
 * in petscksp.h.  Matrices follow AIJ INSERT_VALUES semantics (a repeated (row, col)
 * overwrites) and keep their columns sorted per row, as PETSc's AIJ format does, so
 * MatMult sums in column order.
 */
#include "petscksp.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <vector>

extern "C" {
#include "../gmres_petsc.h"
}

struct _p_Vec {
  std::vector<double> a;
};
struct _p_Mat {
  int n = 0;
  std::vector<std::map<int, double>> rows;
  std::vector<std::vector<int>> log;  /* columns of every MatSetValues per row, in call order */
  std::vector<int> rp, ci;
  std::vector<double> v;
};
struct _p_PC {
  int jacobi = 0;
};
struct _p_KSP {
  Mat A = nullptr;
  _p_PC pc;
  oracle_gmres_params prm;
};
struct _p_VecScatter {
  int dummy = 0;
};

namespace {
oracle_gmres_params g_opts = {30, 1e-5, 1e-50, 1e5, 10000, 0, 0.0, 0, 1};
struct SolveStat {
  int its;
  double rnorm;
  int reason;
  double seconds;
};
std::vector<SolveStat> g_stats;
Mat g_last[2] = {nullptr, nullptr};
int g_mat_counter = 0;
std::vector<int> g_keep_rp[2], g_keep_ci[2];
std::vector<double> g_keep_v[2];
int g_keep_n[2] = {0, 0};
/* insertion order of the kept matrices: Build_Linear_System sets A1's row i as the lm
   stencil neighbours in search order, then the diagonal (solver.cpp:116-125), so the log
   of A1 is the reference's own stencil of every cell */
std::vector<int> g_keep_log_rp[2], g_keep_log_ci[2];
}  // namespace

extern "C" void petsc_shim_set_options(int restart, double rtol, double atol, double dtol, int max_it) {
  g_opts.restart = restart;
  g_opts.rtol = rtol;
  g_opts.atol = atol;
  g_opts.dtol = dtol;
  g_opts.max_it = max_it;
}
extern "C" void petsc_shim_set_threads(int threads) { g_opts.threads = threads > 1 ? threads : 1; }
extern "C" int petsc_shim_solve_count(void) { return (int)g_stats.size(); }
extern "C" void petsc_shim_solve_stats(int k, int *its, double *rnorm, int *reason, double *sec) {
  if (k < 0 || k >= (int)g_stats.size()) return;
  *its = g_stats[k].its;
  *rnorm = g_stats[k].rnorm;
  *reason = g_stats[k].reason;
  *sec = g_stats[k].seconds;
}
extern "C" void petsc_shim_reset_stats(void) { g_stats.clear(); }
extern "C" int petsc_shim_last_matrix(int which, int *n, int *nnz, const int **rp, const int **ci,
                                      const double **v) {
  if (which < 0 || which > 1) return -1;
  *n = g_keep_n[which];
  *nnz = (int)g_keep_v[which].size();
  *rp = g_keep_rp[which].data();
  *ci = g_keep_ci[which].data();
  *v = g_keep_v[which].data();
  return 0;
}
extern "C" int petsc_shim_last_matrix_log(int which, int *n, int *len, const int **rp, const int **ci) {
  if (which < 0 || which > 1) return -1;
  *n = g_keep_n[which];
  *len = (int)g_keep_log_ci[which].size();
  *rp = g_keep_log_rp[which].data();
  *ci = g_keep_log_ci[which].data();
  return 0;
}

int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
int MPI_Barrier(MPI_Comm) { return 0; }
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }

PetscErrorCode VecCreate(MPI_Comm, Vec *v) { *v = new _p_Vec(); return 0; }
PetscErrorCode VecSetSizes(Vec v, PetscInt, PetscInt N) { v->a.assign(N, 0.0); return 0; }
PetscErrorCode VecSetFromOptions(Vec) { return 0; }
PetscErrorCode VecDuplicate(Vec v, Vec *w) { *w = new _p_Vec(); (*w)->a.assign(v->a.size(), 0.0); return 0; }
PetscErrorCode VecSetValues(Vec v, PetscInt ni, const PetscInt ix[], const PetscScalar y[], InsertMode) {
  for (int k = 0; k < ni; ++k) {
    if (ix[k] < 0 || ix[k] >= (int)v->a.size()) return 63;
    v->a[ix[k]] = y[k];
  }
  return 0;
}
PetscErrorCode VecGetValues(Vec v, PetscInt ni, const PetscInt ix[], PetscScalar y[]) {
  for (int k = 0; k < ni; ++k) {
    if (ix[k] < 0 || ix[k] >= (int)v->a.size()) return 63;
    y[k] = v->a[ix[k]];
  }
  return 0;
}
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
PetscErrorCode VecGetArray(Vec v, PetscScalar **p) { *p = v->a.data(); return 0; }
PetscErrorCode VecRestoreArray(Vec, PetscScalar **p) { *p = nullptr; return 0; }
PetscErrorCode VecDestroy(Vec *v) { delete *v; *v = nullptr; return 0; }
PetscErrorCode VecScatterCreateToZero(Vec v, VecScatter *ctx, Vec *out) {
  *ctx = new _p_VecScatter();
  *out = new _p_Vec();
  (*out)->a.assign(v->a.size(), 0.0);
  return 0;
}
PetscErrorCode VecScatterBegin(VecScatter, Vec x, Vec y, InsertMode, ScatterMode) {
  y->a = x->a;
  return 0;
}
PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode) { return 0; }
PetscErrorCode VecScatterDestroy(VecScatter *c) { delete *c; *c = nullptr; return 0; }

PetscErrorCode MatCreate(MPI_Comm, Mat *m) { *m = new _p_Mat(); return 0; }
PetscErrorCode MatSetSizes(Mat m, PetscInt, PetscInt, PetscInt M, PetscInt) {
  m->n = M;
  m->rows.assign(M, {});
  m->log.assign(M, {});
  return 0;
}
PetscErrorCode MatSetFromOptions(Mat) { return 0; }
PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt[], PetscInt, const PetscInt[]) { return 0; }
PetscErrorCode MatSeqAIJSetPreallocation(Mat, PetscInt, const PetscInt[]) { return 0; }
PetscErrorCode MatSetUp(Mat) { return 0; }
PetscErrorCode MatSetValues(Mat m, PetscInt nr, const PetscInt ir[], PetscInt nc, const PetscInt ic[],
                            const PetscScalar v[], InsertMode) {
  for (int a = 0; a < nr; ++a)
    for (int b = 0; b < nc; ++b) {
      if (ir[a] < 0 || ir[a] >= m->n || ic[b] < 0 || ic[b] >= m->n) return 63;
      m->rows[ir[a]][ic[b]] = v[a * nc + b];
      m->log[ir[a]].push_back(ic[b]);
    }
  return 0;
}
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat m, MatAssemblyType) {
  m->rp.assign(m->n + 1, 0);
  m->ci.clear();
  m->v.clear();
  for (int i = 0; i < m->n; ++i) {
    for (auto &kv : m->rows[i]) {
      m->ci.push_back(kv.first);
      m->v.push_back(kv.second);
    }
    m->rp[i + 1] = (int)m->ci.size();
  }
  /* keep copies of the two most recent matrices (A1 then A2 per Build_Linear_System) */
  int slot = g_mat_counter++ & 1;
  g_keep_n[slot] = m->n;
  g_keep_rp[slot] = m->rp;
  g_keep_ci[slot] = m->ci;
  g_keep_v[slot] = m->v;
  g_keep_log_rp[slot].assign(m->n + 1, 0);
  g_keep_log_ci[slot].clear();
  for (int i = 0; i < m->n; ++i) {
    g_keep_log_ci[slot].insert(g_keep_log_ci[slot].end(), m->log[i].begin(), m->log[i].end());
    g_keep_log_rp[slot][i + 1] = (int)g_keep_log_ci[slot].size();
  }
  return 0;
}
PetscErrorCode MatDestroy(Mat *m) { delete *m; *m = nullptr; return 0; }

PetscErrorCode KSPCreate(MPI_Comm, KSP *k) { *k = new _p_KSP(); oracle_gmres_defaults(&(*k)->prm); return 0; }
PetscErrorCode KSPSetType(KSP, KSPType) { return 0; }
PetscErrorCode KSPSetOperators(KSP k, Mat A, Mat) { k->A = A; return 0; }
PetscErrorCode KSPGetPC(KSP k, PC *pc) { *pc = &k->pc; return 0; }
PetscErrorCode PCSetType(PC pc, PCType t) { pc->jacobi = std::strcmp(t, PCJACOBI) == 0; return 0; }
PetscErrorCode KSPSetFromOptions(KSP k) {
  k->prm.restart = g_opts.restart;
  k->prm.rtol = g_opts.rtol;
  k->prm.atol = g_opts.atol;
  k->prm.dtol = g_opts.dtol;
  k->prm.max_it = g_opts.max_it;
  k->prm.threads = g_opts.threads;
  return 0;
}
PetscErrorCode KSPSetUp(KSP) { return 0; }
PetscErrorCode KSPSolve(KSP k, Vec b, Vec x) {
  Mat A = k->A;
  x->a.assign(A->n, 0.0);
  auto t0 = std::chrono::steady_clock::now();
  int rc = oracle_gmres_csr(A->n, A->rp.data(), A->ci.data(), A->v.data(), b->a.data(), x->a.data(), &k->prm);
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  g_stats.push_back({k->prm.its, k->prm.rnorm, k->prm.reason, sec});
  return rc ? 55 : 0;
}
PetscErrorCode KSPDestroy(KSP *k) { delete *k; *k = nullptr; return 0; }
