/*
 * Shared state of the reference's Mover and Solver when their bodies run on
 * libapcloud_gpu.so (mover_gpu.cpp, solver_gpu.cpp).
 *
 * The reference's classes keep their declarations (mover.h:10-44, solver.h:12-64), so the
 * GPU context cannot be a member.  Mover and Solver of one simulation share the
 * Computational_particle they were constructed with (test.cpp:58-66); the context is
 * looked up by that pointer.  The Solver's command line (the -ksp_* options that PETSc
 * would read, solver.cpp:202, 275) is recorded the same way and applied when the Mover's
 * first selection creates the context.
 */
#ifndef APC_DROPIN_H
#define APC_DROPIN_H

#include "apcloud_gpu.h"
#include "particle.h"

struct apc_dropin_entry {
  apc_context *ctx;
  int argc;
  char **argv;
};

/* the entry of a Computational_particle (created empty on first use) */
apc_dropin_entry *apc_dropin_lookup(const Computational_particle *cp);
/* destroy the entry's context and forget it */
void apc_dropin_release(const Computational_particle *cp);

extern "C" {
/* precision of contexts created from now on (apc_precision; default APC_PREC_FP64, the
   reference's GMRES semantics) */
void apc_dropin_set_precision(int precision);
/* how many Mover::move_velocity calls (Controller steps) ran since the last reset */
long apc_dropin_kicks(void);
void apc_dropin_reset_kicks(void);
}

#endif
