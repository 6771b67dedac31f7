/*
 * The reference's Solver (solver.h) with its bodies on libapcloud_gpu.so: GFD assembly,
 * the density and potential solves and the differentiation (solver.cpp:24-454) run on the
 * B200 through apc_solve.  Compiled against the reference's own solver.h, it replaces
 * solver.cpp in the reference's build.  The solves read the -ksp_* options of the
 * command line given to the constructor, as KSPSetFromOptions does (solver.cpp:202, 275).
 * After a solve the Computational_particle's Density, Potential and p_x .. p_yz hold the
 * results, as after the reference's Solve_Density / Solve_Potential / Differentiate.
 */
#include <cstdio>

#include "apc_dropin.h"
#include "solver.h"

Solver::Solver(Computational_particle *computational_particle1, int argc_o, char *args_o[])
    : cp(computational_particle1), argc(argc_o), args(args_o) {
  // the reference's defaults (solver.cpp:8-18)
  BC = 1;
  Constant_For_Density_Estimator = 1.0;
  Constant_For_Potential_Solver = 1.0;
  Constant_For_Field_Solver = 1.0;
  lm = 17;
  ln = 9;
  dirichlet_point = 1;
  apc_dropin_entry *e = apc_dropin_lookup(cp);
  e->argc = argc;
  e->argv = args;
}

Solver::~Solver() {}

int Solver::solve() {
  apc_dropin_entry *e = apc_dropin_lookup(cp);
  if (!e->ctx) {
    std::fprintf(stderr, "Solver::solve: no selection yet\n");
    return 1;
  }
  int rc = apc_solve(e->ctx, Constant_For_Density_Estimator, Constant_For_Potential_Solver, Constant_For_Field_Solver);
  if (rc != APC_OK) {
    std::fprintf(stderr, "apc_solve: %s (%s)\n", apc_status_string(rc), apc_last_error(e->ctx));
    return 1;
  }
  const int M = cp->nc + cp->nv;
  std::vector<double> d9((size_t)M * 9);
  cp->Density.resize(M);
  cp->Potential.resize(M);
  rc = apc_get_fields(e->ctx, cp->Density.data(), cp->Potential.data(), d9.data());
  if (rc != APC_OK) return 1;
  std::vector<double> *out[9] = {&cp->p_x, &cp->p_y, &cp->p_z, &cp->p_xx, &cp->p_yy, &cp->p_zz,
                                 &cp->p_xy, &cp->p_xz, &cp->p_yz};
  for (int k = 0; k < 9; ++k) {
    out[k]->resize(M);
    for (int i = 0; i < M; ++i) (*out[k])[i] = d9[(size_t)i * 9 + k];
  }
  return 0;
}
