/*
 * Test infrastructure (oracle): plain-C restatement of the reference's per-step
 * gravity path (octree build, selection, GFD solver, mover).  It is the checker for
 * the CUDA path; it is never linked into, loaded by, or called from the product.
 *
 * The handle API mirrors the harness around the reference (ref_harness.cpp) so the
 * same tests drive both: apcor_* here, apcref_* there.
 */
#ifndef APC_ORACLE_H
#define APC_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

void *apcor_create(int n, const double *x, const double *y, const double *z, const double *vx,
                   const double *vy, const double *vz, int depth, int bc, const double *box,
                   double gfd_c, int lm);
void apcor_destroy(void *h);
void apcor_set_gmres(int restart, double rtol, double atol, double dtol, int max_it);
void apcor_set_maxnc(void *h, int maxnc);
int apcor_select(void *h);
int apcor_cell_counts(void *h, int *nc, int *nv, int *nb, int *nneigh);
int apcor_get_cells(void *h, double *x, double *y, double *z, double *len, int *first, int *count,
                    int *type, int *firstneigh, int *numneigh, int *neigh24);
int apcor_get_keys(void *h, uint64_t *keys, int *index);
int apcor_octree_levels(void *h, int *numnodes);
int apcor_solve(void *h, double c_dens, double c_pot, double c_field);
int apcor_get_fields(void *h, double *density, double *potential, double *deriv9);
/* Solver::Differentiate (solver.cpp:295-362) of the given potential on the selected cells
 * (after apcor_select); returns 0 or the search / least-squares failure code */
int apcor_differentiate(void *h, const double *potential, double c_field, double *deriv9);
int apcor_get_stencils(void *h, int *idx17, double *dist17);
int apcor_solve_stats(int k, int *its, double *rnorm, int *reason, double *seconds);
int apcor_solve_count(void);
void apcor_reset_solve_stats(void);
int apcor_last_matrix(int which, int *n, int *nnz, int *rp, int *ci, double *v);
double apcor_move_velocity(void *h, double dt, double c_vel);
double apcor_move_position(void *h, double dt, double c_pos);
int apcor_get_particles(void *h, double *x, double *y, double *z, double *vx, double *vy,
                        double *vz, double *ax, double *ay, double *az);
void apcor_phase_times(void *h, double *t3);

/* Morton key of one point (octree.cpp:676-852), exposed for unit tests */
uint64_t apcor_key64(double x, double y, double z, const double *box, int depth);

#ifdef __cplusplus
}
#endif
#endif
