/*
 * Test infrastructure (oracle): single-rank stand-in for the slice of the PETSc 3.5
 * API that the reference's solver.cpp uses, so that the reference's own solver.cpp
 * compiles and runs here (PETSc is not vendored in the reference and not installed).
 *
 * Implemented calls: exactly those at solver.cpp:36-64, 122-178, 194-216, 262-291,
 * 364-380 (Vec/Mat/KSP/PC/VecScatter) and the MPI calls at solver.cpp:30-31,410,424.
 * KSPSolve runs oracle_gmres_csr (PETSc-3.5 GMRES semantics, gmres_petsc.c).
 * KSPSetFromOptions reads the process-wide options set by petsc_shim_set_options,
 * standing in for the -ksp_* command-line flags of the reference's run lines.
 */
#ifndef APC_SHIM_PETSCKSP_H
#define APC_SHIM_PETSCKSP_H

#include <cstddef>

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int InsertMode;
typedef int ScatterMode;
typedef int MatAssemblyType;
typedef const char *KSPType;
typedef const char *PCType;

#define PETSC_COMM_WORLD 0
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define PETSC_DECIDE (-1)
#define PETSC_TRUE 1
#define PETSC_FALSE 0
#define INSERT_VALUES 1
#define SCATTER_FORWARD 0
#define MAT_FINAL_ASSEMBLY 0
#define KSPGMRES "gmres"
#define PCJACOBI "jacobi"
#define CHKERRQ(e) do { if (e) return (e); } while (0)

struct _p_Vec;
struct _p_Mat;
struct _p_KSP;
struct _p_PC;
struct _p_VecScatter;
typedef _p_Vec *Vec;
typedef _p_Mat *Mat;
typedef _p_KSP *KSP;
typedef _p_PC *PC;
typedef _p_VecScatter *VecScatter;

int MPI_Comm_rank(MPI_Comm, int *rank);
int MPI_Comm_size(MPI_Comm, int *size);
int MPI_Barrier(MPI_Comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm);

PetscErrorCode VecCreate(MPI_Comm, Vec *);
PetscErrorCode VecSetSizes(Vec, PetscInt n, PetscInt N);
PetscErrorCode VecSetFromOptions(Vec);
PetscErrorCode VecDuplicate(Vec, Vec *);
PetscErrorCode VecSetValues(Vec, PetscInt ni, const PetscInt ix[], const PetscScalar y[], InsertMode);
PetscErrorCode VecGetValues(Vec, PetscInt ni, const PetscInt ix[], PetscScalar y[]);
PetscErrorCode VecAssemblyBegin(Vec);
PetscErrorCode VecAssemblyEnd(Vec);
PetscErrorCode VecGetArray(Vec, PetscScalar **);
PetscErrorCode VecRestoreArray(Vec, PetscScalar **);
PetscErrorCode VecDestroy(Vec *);
PetscErrorCode VecScatterCreateToZero(Vec, VecScatter *, Vec *);
PetscErrorCode VecScatterBegin(VecScatter, Vec, Vec, InsertMode, ScatterMode);
PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode);
PetscErrorCode VecScatterDestroy(VecScatter *);

PetscErrorCode MatCreate(MPI_Comm, Mat *);
PetscErrorCode MatSetSizes(Mat, PetscInt m, PetscInt n, PetscInt M, PetscInt N);
PetscErrorCode MatSetFromOptions(Mat);
PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt[], PetscInt, const PetscInt[]);
PetscErrorCode MatSeqAIJSetPreallocation(Mat, PetscInt, const PetscInt[]);
PetscErrorCode MatSetUp(Mat);
PetscErrorCode MatSetValues(Mat, PetscInt m, const PetscInt idxm[], PetscInt n, const PetscInt idxn[],
                            const PetscScalar v[], InsertMode);
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType);
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType);
PetscErrorCode MatDestroy(Mat *);

PetscErrorCode KSPCreate(MPI_Comm, KSP *);
PetscErrorCode KSPSetType(KSP, KSPType);
PetscErrorCode KSPSetOperators(KSP, Mat, Mat);
PetscErrorCode KSPGetPC(KSP, PC *);
PetscErrorCode PCSetType(PC, PCType);
PetscErrorCode KSPSetFromOptions(KSP);
PetscErrorCode KSPSetUp(KSP);
PetscErrorCode KSPSolve(KSP, Vec b, Vec x);
PetscErrorCode KSPDestroy(KSP *);

/* ---- shim control (not PETSc API) ---- */
extern "C" {
void petsc_shim_set_options(int restart, double rtol, double atol, double dtol, int max_it);
/* statistics of the most recent KSPSolve calls, in call order (density, potential) */
int petsc_shim_solve_count(void);
void petsc_shim_solve_stats(int k, int *its, double *rnorm, int *reason, double *seconds);
void petsc_shim_reset_stats(void);
/* the most recently assembled matrices in CSR form (for parity tests) */
int petsc_shim_last_matrix(int which, int *n, int *nnz, const int **rowptr, const int **col,
                           const double **val);
/* the columns of every MatSetValues call on those matrices, per row in call order */
int petsc_shim_last_matrix_log(int which, int *n, int *len, const int **rowptr, const int **col);
/* host threads of the GMRES shim's vector and matrix loops (1 = serial, the default; the
   serial order is the one the parity tests pin) */
void petsc_shim_set_threads(int threads);
}

#endif
