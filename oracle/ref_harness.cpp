/*
 * Test infrastructure (oracle): C API around the REFERENCE's own classes, compiled
 * from the reference sources by oracle/Makefile into oracle/_ref/libapcref.so.
 * Used to pin the oracle restatement and as the timed CPU baseline; never part of
 * the product library.
 *
 * The harness drives the reference only through its public interface (Octree,
 * Mover, Solver setters and phase calls, octree.h:224-251, mover.h:31-43,
 * solver.h:53-62) and replays the step sequence of Controller::solve
 * (controller.cpp:54-241) with:
 *   - adaptive time stepping off (ADAPTIVE_TIME_STEP, apcloud_macro.h:25-27);
 *   - viewer output off (controller.cpp:122-131);
 *   - the constants passed per phase by the caller (controller.cpp:182-186).
 * Internals (sorted keys, octree levels) are read for parity checks through
 * `private`-to-`public` access, without changing any reference code.
 */
#include <pthread.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
/* every system header the reference headers pull in, so that the access override
 * below reaches only the reference's own classes */
#include <omp.h>
#include <stdint.h>
#include <algorithm>
#include <ctime>
#include <cstdlib>
#include <deque>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <math.h>
#include <numeric>
#include "lapacke.h"
#include "petscksp.h"
#include "particle.h"
#include "parameter.h"

#define private public
#include "octree.h"
#include "mover.h"
#include "solver.h"
#undef private

#include "petscksp.h"

namespace {
struct Ref {
  Physical_particle pp;
  Computational_particle cp;
  Mover *mover = nullptr;
  Solver *solver = nullptr;
  int depth = 20, bc = 1, lm = 17;
  double box[6] = {0, 1, 0, 1, 0, 1};
  double gfd_c = 0.0;
  int last_select = -1;
  double t_select = 0, t_solve = 0, t_move = 0;
};

template <class F>
struct ThreadCall {
  F *f;
  static void *run(void *p) {
    (*static_cast<ThreadCall *>(p)->f)();
    return nullptr;
  }
};

/* The reference's selection keeps its temporary node arrays in stack VLAs sized by
 * nmax (octree.cpp:1112-1113); run it on a thread with a 2 GiB stack so that the
 * Python host's default 8 MiB stack limit does not apply. */
template <class F>
void run_on_big_stack(F f) {
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, (size_t)2 << 30);
  pthread_t th;
  ThreadCall<F> tc{&f};
  if (pthread_create(&th, &attr, &ThreadCall<F>::run, &tc) != 0) {
    f();
  } else {
    pthread_join(th, nullptr);
  }
  pthread_attr_destroy(&attr);
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

extern "C" {

void *apcref_create(int n, const double *x, const double *y, const double *z, const double *vx,
                    const double *vy, const double *vz, int depth, int bc, const double *box,
                    double gfd_c, int lm) {
  Ref *r = new Ref();
  r->pp.size = n;
  r->pp.x = new double[n];
  r->pp.y = new double[n];
  r->pp.z = new double[n];
  r->pp.v_x = new double[n];
  r->pp.v_y = new double[n];
  r->pp.v_z = new double[n];
  r->pp.a_x = new double[n];
  r->pp.a_y = new double[n];
  r->pp.a_z = new double[n];
  r->pp.ID = new int[n];
  r->pp.mass = nullptr;
  r->pp.uniform_mass = 1.0 / n;
  for (int i = 0; i < n; ++i) {
    r->pp.x[i] = x[i];
    r->pp.y[i] = y[i];
    r->pp.z[i] = z[i];
    r->pp.v_x[i] = vx[i];
    r->pp.v_y[i] = vy[i];
    r->pp.v_z[i] = vz[i];
    r->pp.a_x[i] = r->pp.a_y[i] = r->pp.a_z[i] = 0.0;
    r->pp.ID[i] = i;
  }
  r->depth = depth;
  r->bc = bc;
  r->lm = lm;
  r->gfd_c = gfd_c;
  for (int k = 0; k < 6; ++k) r->box[k] = box[k];
  r->cp.size = r->cp.nc = r->cp.nv = r->cp.nb = 0;
  /* test.cpp:58-62 construct order; controller.cpp:75-81 mover setup */
  r->solver = new Solver(&r->cp, 0, nullptr);
  r->mover = new Mover(&r->pp, &r->cp);
  r->mover->Set_BoundingBox(box[0], box[1], box[2], box[3], box[4], box[5]);
  r->mover->Set_maxnc(10000);
  r->mover->Set_Octree_Depth(depth);
  r->mover->Set_Constant_For_GFD_Constant(gfd_c);
  r->mover->Set_BC(bc);
  /* controller.cpp:99-101 solver setup */
  r->solver->Set_BoundingBox(box[0], box[1], box[2], box[3], box[4], box[5]);
  r->solver->Set_Boundary_Condition(bc);
  r->solver->Set_NumberOfGFDNeighbors(lm);
  return r;
}

void apcref_destroy(void *h) {
  Ref *r = static_cast<Ref *>(h);
  if (!r) return;
  if (r->mover->octree) r->mover->octree->~Octree();
  r->mover->octree = nullptr;
  operator delete(static_cast<void *>(r->mover)); /* Mover's dtor dereferences octree unconditionally (mover.cpp:12-15) */
  delete r->solver;
  delete[] r->pp.x; delete[] r->pp.y; delete[] r->pp.z;
  delete[] r->pp.v_x; delete[] r->pp.v_y; delete[] r->pp.v_z;
  delete[] r->pp.a_x; delete[] r->pp.a_y; delete[] r->pp.a_z;
  delete[] r->pp.ID;
  delete r;
}

void apcref_set_gmres(int restart, double rtol, double atol, double dtol, int max_it) {
  petsc_shim_set_options(restart, rtol, atol, dtol, max_it);
}

void apcref_set_maxnc(void *h, int maxnc) { static_cast<Ref *>(h)->mover->Set_maxnc(maxnc); }

/* Mover::select_computational_particles (mover.cpp:17-49): octree build + selection */
int apcref_select(void *h) {
  Ref *r = static_cast<Ref *>(h);
  double t0 = now();
  run_on_big_stack([r]() { r->last_select = r->mover->select_computational_particles(); });
  r->t_select += now() - t0;
  return r->last_select;
}

int apcref_cell_counts(void *h, int *nc, int *nv, int *nb, int *nneigh) {
  Ref *r = static_cast<Ref *>(h);
  *nc = r->cp.nc;
  *nv = r->cp.nv;
  *nb = r->cp.nb;
  *nneigh = (int)r->cp.Neigh24.size();
  return r->cp.size;
}

int apcref_get_cells(void *h, double *x, double *y, double *z, double *len, int *first, int *count,
                     int *type, int *firstneigh, int *numneigh, int *neigh24) {
  Ref *r = static_cast<Ref *>(h);
  int m = r->cp.size;
  for (int i = 0; i < m; ++i) {
    x[i] = r->cp.x[i];
    y[i] = r->cp.y[i];
    z[i] = r->cp.z[i];
    len[i] = r->cp.CellLength[i];
    first[i] = r->cp.IndexOfFirstPhysicalParticle[i];
    count[i] = r->cp.NumberOfPhysicalParticles[i];
    type[i] = r->cp.Type[i];
    firstneigh[i] = r->cp.FirstNeigh[i];
    numneigh[i] = r->cp.NumberNeigh[i];
  }
  for (size_t k = 0; k < r->cp.Neigh24.size(); ++k) neigh24[k] = r->cp.Neigh24[k];
  return m;
}

/* sorted (key, index) pairs of the current octree (octree.cpp:131-148) */
int apcref_get_keys(void *h, uint64_t *keys, int *index) {
  Ref *r = static_cast<Ref *>(h);
  Octree *o = r->mover->octree;
  if (!o) return -1;
  for (int i = 0; i < o->m_iTotalNumberOfParticles; ++i) {
    keys[i] = o->m_vParticleKeyIndex[i].key;
    index[i] = o->m_vParticleKeyIndex[i].index;
  }
  return o->m_iTotalNumberOfParticles;
}

/* per-level node counts numnodes[0..depth] (octree.cpp:174-191), recovered from m_vDepth */
int apcref_octree_levels(void *h, int *numnodes) {
  Ref *r = static_cast<Ref *>(h);
  Octree *o = r->mover->octree;
  if (!o) return -1;
  for (int k = 0; k <= o->m_iMaxDepth; ++k) numnodes[k] = 0;
  for (int i = 0; i < o->m_iTreeLength; ++i) numnodes[o->m_vDepth[i]]++;
  return o->m_iTreeLength;
}

/* full octree node arrays (octree.cpp:217-313), BFS by level, key order within level */
int apcref_octree_nodes(void *h, uint64_t *key, int *depth, int *first, int *count, int *firstchild,
                        int *nchild) {
  Ref *r = static_cast<Ref *>(h);
  Octree *o = r->mover->octree;
  if (!o) return -1;
  for (int i = 0; i < o->m_iTreeLength; ++i) {
    key[i] = o->m_vNodeKey[i];
    depth[i] = o->m_vDepth[i];
    first[i] = o->m_vFirstParticleIndex[i];
    count[i] = o->m_vNumberOfContainedParticles[i];
    firstchild[i] = o->m_vFirstChildIndex[i];
    nchild[i] = o->m_vNumberOfChildren[i];
  }
  return o->m_iTreeLength;
}

/* Solver::solve (solver.cpp:382-454) with the constants of controller.cpp:184-186 */
int apcref_solve(void *h, double c_dens, double c_pot, double c_field) {
  Ref *r = static_cast<Ref *>(h);
  r->solver->Set_Constant_For_Density_Estimator(c_dens);
  r->solver->Set_Constant_For_Potential_Solver(c_pot);
  r->solver->Set_Constant_For_Field_Solver(c_field);
  double t0 = now();
  int rc = r->solver->solve();
  r->t_solve += now() - t0;
  return rc;
}

int apcref_get_fields(void *h, double *density, double *potential, double *deriv9) {
  Ref *r = static_cast<Ref *>(h);
  int m = r->cp.nc + r->cp.nv;
  for (int i = 0; i < m; ++i) {
    density[i] = r->cp.Density[i];
    potential[i] = r->cp.Potential[i];
    deriv9[9 * i + 0] = r->cp.p_x[i];
    deriv9[9 * i + 1] = r->cp.p_y[i];
    deriv9[9 * i + 2] = r->cp.p_z[i];
    deriv9[9 * i + 3] = r->cp.p_xx[i];
    deriv9[9 * i + 4] = r->cp.p_yy[i];
    deriv9[9 * i + 5] = r->cp.p_zz[i];
    deriv9[9 * i + 6] = r->cp.p_xy[i];
    deriv9[9 * i + 7] = r->cp.p_xz[i];
    deriv9[9 * i + 8] = r->cp.p_yz[i];
  }
  return m;
}

int apcref_solve_stats(int k, int *its, double *rnorm, int *reason, double *seconds) {
  if (k >= petsc_shim_solve_count()) return -1;
  petsc_shim_solve_stats(k, its, rnorm, reason, seconds);
  return 0;
}
int apcref_solve_count(void) { return petsc_shim_solve_count(); }
void apcref_reset_solve_stats(void) { petsc_shim_reset_stats(); }

int apcref_last_matrix(int which, int *n, int *nnz, int *rp, int *ci, double *v) {
  const int *a, *b;
  const double *c;
  int nn, nz;
  if (petsc_shim_last_matrix(which, &nn, &nz, &a, &b, &c)) return -1;
  if (n) *n = nn;
  if (nnz) *nnz = nz;
  if (rp) std::memcpy(rp, a, sizeof(int) * (nn + 1));
  if (ci) std::memcpy(ci, b, sizeof(int) * nz);
  if (v) std::memcpy(v, c, sizeof(double) * nz);
  return 0;
}

/* The GFD stencil of every cell of the last solve, lm indices per cell in search order:
 * Build_Linear_System inserts row i of A1 as its lm neighbours in the order
 * searchneighboroctant returned them, then the diagonal (solver.cpp:116-125), so the
 * first lm columns of each row's insertion log are the reference's own stencil. */
int apcref_get_stencils(int lm, int *idx) {
  const int *rp, *ci;
  int n, len;
  if (petsc_shim_last_matrix_log(0, &n, &len, &rp, &ci)) return -1;
  for (int i = 0; i < n; ++i) {
    if (rp[i + 1] - rp[i] < lm) return -1;
    for (int j = 0; j < lm; ++j) idx[(size_t)i * lm + j] = ci[rp[i] + j];
  }
  return n;
}

/* host threads of the GMRES shim (PETSc spreads its solves over MPI ranks) */
void apcref_set_threads(int threads) { petsc_shim_set_threads(threads); }

/* Mover::move_velocity (mover.cpp:51-89): interpolation + kick */
double apcref_move_velocity(void *h, double dt, double c_vel) {
  Ref *r = static_cast<Ref *>(h);
  r->mover->Set_Constant_For_Mover_Velocity(c_vel);
  double t0 = now();
  double d = r->mover->move_velocity(dt);
  r->t_move += now() - t0;
  return d;
}

/* Mover::move_position (mover.cpp:91-121): drift + periodic wrap */
double apcref_move_position(void *h, double dt, double c_pos) {
  Ref *r = static_cast<Ref *>(h);
  r->mover->Set_Constant_For_Mover_Position(c_pos);
  double t0 = now();
  double d = r->mover->move_position(dt);
  r->t_move += now() - t0;
  return d;
}

int apcref_get_particles(void *h, double *x, double *y, double *z, double *vx, double *vy, double *vz,
                         double *ax, double *ay, double *az) {
  Ref *r = static_cast<Ref *>(h);
  int n = r->pp.size;
  for (int i = 0; i < n; ++i) {
    if (x) x[i] = r->pp.x[i];
    if (y) y[i] = r->pp.y[i];
    if (z) z[i] = r->pp.z[i];
    if (vx) vx[i] = r->pp.v_x[i];
    if (vy) vy[i] = r->pp.v_y[i];
    if (vz) vz[i] = r->pp.v_z[i];
    if (ax) ax[i] = r->pp.a_x[i];
    if (ay) ay[i] = r->pp.a_y[i];
    if (az) az[i] = r->pp.a_z[i];
  }
  return n;
}

void apcref_phase_times(void *h, double *t3) {
  Ref *r = static_cast<Ref *>(h);
  t3[0] = r->t_select;
  t3[1] = r->t_solve;
  t3[2] = r->t_move;
}

}  // extern "C"
