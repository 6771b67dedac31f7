/*
 * Runs the reference's own Controller::solve (controller.cpp:54-241) on a particle set
 * given by the caller, with the reference's construction sequence (test.cpp:58-66):
 * Solver(cp, argc, argv), Viewer(pp, cp), Mover(pp, cp), Controller(...).  Which Mover and
 * Solver bodies run is decided at link time: this file is linked with mover_gpu.cpp /
 * solver_gpu.cpp into the GPU build, and with the reference's mover.cpp / solver.cpp /
 * octree.cpp into the CPU build that checks it.  The viewer is linked with output off.
 *
 * The Controller runs with the reference's macros (apcloud_macro.h: adaptive time step on,
 * COSMOLOGY_UNIT off) and its -ksp_* options come from the command line, as in the
 * reference's run lines (Makefile:30-32).
 */
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "controller.h"

#ifdef APC_DROPIN_CPU
extern "C" void petsc_shim_set_options(int restart, double rtol, double atol, double dtol, int max_it);
#endif

extern "C" int apc_dropin_run(int n, double *x, double *y, double *z, double *vx, double *vy, double *vz,
                              double *ax, double *ay, double *az, double start_a, double end_a, double delta_a,
                              int depth, double gfd_c, int lm, const double *box, int gmres_restart,
                              double gmres_rtol, int gmres_max_it) {
  // the -ksp_* options of a reference run line
  std::vector<std::string> words = {"apcloud", "parameter.param", "-ksp_gmres_restart", std::to_string(gmres_restart),
                                    "-ksp_rtol", std::to_string(gmres_rtol), "-ksp_max_it",
                                    std::to_string(gmres_max_it)};
  char rtol_text[64];
  std::snprintf(rtol_text, sizeof(rtol_text), "%.17g", gmres_rtol);
  words[5] = rtol_text;
  std::vector<char *> argv;
  for (auto &w : words) argv.push_back(&w[0]);
  argv.push_back(nullptr);
  const int argc = (int)words.size();
#ifdef APC_DROPIN_CPU
  // the PETSc shim of the CPU build reads its options here instead of from argv
  petsc_shim_set_options(gmres_restart, gmres_rtol, 1e-50, 1e5, gmres_max_it);
#endif

  Physical_particle pp;
  pp.size = n;
  pp.x = x;
  pp.y = y;
  pp.z = z;
  pp.v_x = vx;
  pp.v_y = vy;
  pp.v_z = vz;
  pp.a_x = ax;
  pp.a_y = ay;
  pp.a_z = az;
  std::vector<int> ids(n);
  for (int i = 0; i < n; ++i) ids[i] = i;
  pp.ID = ids.data();
  pp.mass = nullptr;
  pp.uniform_mass = 1.0 / n;
  for (int i = 0; i < n; ++i) ax[i] = ay[i] = az[i] = 0.0;

  Computational_particle cp;
  cp.size = cp.nc = cp.nv = cp.nb = 0;
  Solver *solver = new Solver(&cp, argc, argv.data());
  Viewer *viewer = new Viewer(&pp, &cp);
  Mover *mover = new Mover(&pp, &cp);
  Controller controller(&pp, &cp, start_a, end_a, delta_a, solver, viewer, mover, 1 << 30, 1, box[0], box[1], box[2],
                        box[3], box[4], box[5], depth, gfd_c, lm);
  const int rc = controller.solve();
  delete mover;
  delete viewer;
  delete solver;
  return rc;
}
