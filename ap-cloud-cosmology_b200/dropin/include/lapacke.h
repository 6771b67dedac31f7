/*
 * Stand-in for lapacke.h in the GPU build of the reference's classes: solver.h includes
 * it (solver.h:2), but the GFD least squares run inside libapcloud_gpu.so, so no LAPACK
 * routine is called on this path and none is declared here.
 */
#ifndef APC_DROPIN_LAPACKE_H
#define APC_DROPIN_LAPACKE_H
#endif
