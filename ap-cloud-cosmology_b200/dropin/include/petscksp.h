/*
 * Stand-in for petscksp.h in the GPU build of the reference's classes.
 *
 * With Mover and Solver running on libapcloud_gpu.so nothing on the per-step path calls
 * PETSc or MPI, yet the reference's headers still name PETSc types (solver.h:36-42) and
 * controller.cpp still broadcasts its step state (controller.cpp:93-96, 176-181, 222).
 * This header declares those types as opaque handles and the MPI calls as the
 * single-rank operations they reduce to, so the reference's controller.cpp, solver.h and
 * mover.h compile unchanged without PETSc or MPI installed.
 */
#ifndef APC_DROPIN_PETSCKSP_H
#define APC_DROPIN_PETSCKSP_H

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef struct _apc_opaque_handle *Mat, *Vec, *KSP, *PC, *VecScatter;

typedef int MPI_Comm;
typedef int MPI_Datatype;
#define PETSC_COMM_WORLD 0
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2

/* one rank: rank 0 of a communicator of size 1; broadcasts and barriers are no-ops */
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }

#endif
