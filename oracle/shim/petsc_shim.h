/*
 * Single-rank stand-in for the subset of the PETSc 3.1 / MPI / HYPRE API that the
 * reference solver's hot-path sources use.  It exists only so that those sources
 * can be compiled unmodified, with g++, into the test oracle (oracle/_ref).  It is
 * test infrastructure: nothing in the product library links or includes it.
 *
 * Semantics emulated (one MPI rank, DA_NONPERIODIC distributed arrays):
 *   - a DA of size mx*my*mz owns every point, so local == global == ghosted extent,
 *     and DAGlobalToLocal / DALocalToGlobal are plain copies, DALocalToLocal a no-op;
 *   - DAVecGetArray returns a T*** view indexable as [k][j][i], exactly like PETSc's
 *     contiguous single-rank storage (an out-of-row index walks into the next row,
 *     as it would in PETSc); a few spare planes before and after the data keep any
 *     stray plane index inside the allocation;
 *   - Mat is a row-map recorder (MatSetValues INSERT/ADD) exportable as CSR;
 *   - KSP / PC / SNES / HYPRE calls are inert stubs (the oracle never solves with them).
 */
#ifndef VFS_PETSC_SHIM_H
#define VFS_PETSC_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdarg.h>

/* ---------------------------------------------------------------- scalars */
typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscReal;
typedef double PetscScalar;
typedef int PetscErrorCode;
typedef long long PetscLogDouble_ll;
typedef double PetscLogDouble;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscTruth;
typedef PetscTruth PetscBool;
typedef int PetscCookie;

#define PETSC_NULL 0
#define PETSC_DECIDE (-1)
#define PETSC_DETERMINE (-1)
#define PETSC_DEFAULT (-2)
#define PETSC_IGNORE 0
#define PETSC_MAX_INT 2147483647

#define PetscMax(a, b) (((a) < (b)) ? (b) : (a))
#define PetscMin(a, b) (((a) < (b)) ? (a) : (b))
#define PetscAbsScalar(a) fabs(a)
#define PetscAbsReal(a) fabs(a)
#define PetscSqrtScalar(a) sqrt(a)
#define PetscRealPart(a) (a)
#define CHKERRQ(e) do { (void)(e); } while (0)
#define SETERRQ(c, s) return (c)
#define PetscFunctionBegin
#define PetscFunctionReturn(x) return (x)

/* ---------------------------------------------------------------- MPI */
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define PETSC_COMM_WORLD 1
#define PETSC_COMM_SELF 2
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPIU_REAL 2
#define MPIU_SCALAR 2
#define MPIU_INT 1
#define MPI_FLOAT 3
#define MPI_CHAR 4
#define MPI_LONG 5
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)

int shim_mpi_type_size(MPI_Datatype t);
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *a, void *b, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (a != b) memmove(b, a, (size_t)n * shim_mpi_type_size(t));
  return 0;
}
static inline int MPI_Reduce(const void *a, void *b, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (a != b) memmove(b, a, (size_t)n * shim_mpi_type_size(t));
  return 0;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Gather(const void *a, int n, MPI_Datatype t, void *b, int, MPI_Datatype, int, MPI_Comm) {
  memmove(b, a, (size_t)n * shim_mpi_type_size(t));
  return 0;
}
static inline int MPI_Allgather(const void *a, int n, MPI_Datatype t, void *b, int, MPI_Datatype, MPI_Comm) {
  memmove(b, a, (size_t)n * shim_mpi_type_size(t));
  return 0;
}
// Derived types and MPI_Gatherv appear only in the reference's sediment-transport code,
// which the oracle driver never runs (that file is compiled for its wall model); a call
// ends the process with the function's name.
extern "C" void shim_unresolved(const char *name);
static inline int MPI_Type_contiguous(int, MPI_Datatype, MPI_Datatype *) { shim_unresolved("MPI_Type_contiguous"); return 1; }
static inline int MPI_Type_commit(MPI_Datatype *) { shim_unresolved("MPI_Type_commit"); return 1; }
static inline int MPI_Gatherv(const void *, int, MPI_Datatype, void *, const int *, const int *, MPI_Datatype, int,
                              MPI_Comm) {
  shim_unresolved("MPI_Gatherv");
  return 1;
}
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
static inline double MPI_Wtime(void) { return 0.0; }

/* ---------------------------------------------------------------- objects */
typedef enum { DA_NONPERIODIC, DA_XPERIODIC, DA_YPERIODIC, DA_XYPERIODIC, DA_XYZPERIODIC,
               DA_XZPERIODIC, DA_YZPERIODIC, DA_ZPERIODIC, DA_XYZGHOSTED } DAPeriodicType;
typedef enum { DA_STENCIL_STAR, DA_STENCIL_BOX } DAStencilType;
typedef enum { INSERT_VALUES, ADD_VALUES, MAX_VALUES } InsertMode;
typedef enum { SCATTER_FORWARD, SCATTER_REVERSE } ScatterMode;
typedef enum { NORM_1, NORM_2, NORM_FROBENIUS, NORM_INFINITY, NORM_1_AND_2 } NormType;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { SAME_NONZERO_PATTERN, DIFFERENT_NONZERO_PATTERN, SAME_PRECONDITIONER,
               SUBSET_NONZERO_PATTERN } MatStructure;
typedef enum { MATOP_MULT, MATOP_MULT_ADD, MATOP_GET_DIAGONAL, MATOP_DESTROY } MatOperation;
typedef enum { KSP_NORM_NO, KSP_NORM_PRECONDITIONED, KSP_NORM_UNPRECONDITIONED,
               KSP_NORM_NATURAL } KSPNormType;
typedef enum { PC_MG_MULTIPLICATIVE, PC_MG_ADDITIVE, PC_MG_FULL, PC_MG_KASKADE } PCMGType;
typedef enum { PC_MG_CYCLE_V = 1, PC_MG_CYCLE_W = 2 } PCMGCycleType;
typedef enum { KSP_CONVERGED_ITERATING = 0 } KSPConvergedReason;
typedef enum { MAT_SHIFT_NONE, MAT_SHIFT_NONZERO, MAT_SHIFT_POSITIVE_DEFINITE,
               MAT_SHIFT_INBLOCKS } MatFactorShiftType;
typedef enum { PETSC_VIEWER_DEFAULT } PetscViewerFormat;
typedef enum { FILE_MODE_READ, FILE_MODE_WRITE, FILE_MODE_APPEND } PetscFileMode;

typedef const char *KSPType;
typedef const char *PCType;
typedef const char *MatType;
typedef const char *SNESType;
#define KSPGMRES "gmres"
#define KSPFGMRES "fgmres"
#define KSPCG "cg"
#define KSPBCGS "bcgs"
#define KSPRICHARDSON "richardson"
#define KSPPREONLY "preonly"
#define KSPCHEBYCHEV "chebychev"
#define PCNONE "none"
#define PCJACOBI "jacobi"
#define PCBJACOBI "bjacobi"
#define PCSOR "sor"
#define PCILU "ilu"
#define PCLU "lu"
#define PCASM "asm"
#define PCMG "mg"
#define PCHYPRE "hypre"
#define PCSHELL "shell"
#define MATMPIAIJ "mpiaij"
#define MATSEQAIJ "seqaij"
#define MATAIJ "aij"
#define SNESTR "tr"
#define SNESLS "ls"

struct _p_DA;
struct _p_Vec;
typedef struct _p_DA *DA;
typedef struct _p_Vec *Vec;
typedef struct _p_Mat *Mat;
typedef void *KSP;
typedef void *PC;
typedef void *SNES;
typedef void *MatNullSpace;
typedef void *VecScatter;
typedef void *IS;
typedef void *AO;
typedef void *PetscViewer;
typedef void *ISLocalToGlobalMapping;
typedef void *MatFDColoring;
typedef void *ISColoring;
typedef void *PetscRandom;

typedef struct {
  PetscInt dim, dof, sw;
  PetscInt mx, my, mz;
  PetscInt xs, ys, zs;
  PetscInt xm, ym, zm;
  PetscInt gxs, gys, gzs;
  PetscInt gxm, gym, gzm;
  DAPeriodicType pt;
  DAStencilType st;
  DA da;
} DALocalInfo;

struct _p_DA {
  PetscInt mx, my, mz, dof, s;
  DA cda;        /* coordinate DA (dof 3) */
  Vec coords;    /* global coordinates */
  Vec gcoords;   /* ghosted coordinates */
  PetscInt *gidx;
};

struct _p_Vec {
  double *data;     /* first owned entry */
  double *base;     /* allocation (with slack) */
  PetscInt n;       /* entries = points * dof */
  DA da;            /* owning DA, or null */
  void **k_table;   /* [k] -> row table, built on first DAVecGetArray */
  void *kj_store;
};

struct shim_csr_row;
struct _p_Mat {
  PetscInt m, n;
  void *rows; /* std::vector<std::map<int,double>> in the implementation */
  void *shell_ctx;
};

/* ---------------------------------------------------------------- DA */
PetscErrorCode DACreate3d(MPI_Comm, DAPeriodicType, DAStencilType, PetscInt M, PetscInt N,
                          PetscInt P, PetscInt m, PetscInt n, PetscInt p, PetscInt dof,
                          PetscInt s, const PetscInt *, const PetscInt *, const PetscInt *,
                          DA *da);
PetscErrorCode DADestroy(DA);
PetscErrorCode DAGetLocalInfo(DA, DALocalInfo *);
PetscErrorCode DAGetInfo(DA, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *,
                         PetscInt *, PetscInt *, PetscInt *, PetscInt *, DAPeriodicType *,
                         DAStencilType *);
PetscErrorCode DAGetCorners(DA, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *,
                            PetscInt *);
PetscErrorCode DAGetGhostCorners(DA, PetscInt *, PetscInt *, PetscInt *, PetscInt *,
                                 PetscInt *, PetscInt *);
PetscErrorCode DACreateGlobalVector(DA, Vec *);
PetscErrorCode DACreateLocalVector(DA, Vec *);
PetscErrorCode DACreateNaturalVector(DA, Vec *);
PetscErrorCode DAGetLocalVector(DA, Vec *);
PetscErrorCode DARestoreLocalVector(DA, Vec *);
PetscErrorCode DAGetGlobalVector(DA, Vec *);
PetscErrorCode DARestoreGlobalVector(DA, Vec *);
PetscErrorCode DAVecGetArray(DA, Vec, void *);
PetscErrorCode DAVecRestoreArray(DA, Vec, void *);
PetscErrorCode DAGlobalToLocalBegin(DA, Vec, InsertMode, Vec);
PetscErrorCode DAGlobalToLocalEnd(DA, Vec, InsertMode, Vec);
PetscErrorCode DALocalToLocalBegin(DA, Vec, InsertMode, Vec);
PetscErrorCode DALocalToLocalEnd(DA, Vec, InsertMode, Vec);
PetscErrorCode DALocalToGlobal(DA, Vec, InsertMode, Vec);
PetscErrorCode DALocalToGlobalBegin(DA, Vec, Vec);
PetscErrorCode DALocalToGlobalEnd(DA, Vec, Vec);
PetscErrorCode DAGlobalToNaturalBegin(DA, Vec, InsertMode, Vec);
PetscErrorCode DAGlobalToNaturalEnd(DA, Vec, InsertMode, Vec);
PetscErrorCode DANaturalToGlobalBegin(DA, Vec, InsertMode, Vec);
PetscErrorCode DANaturalToGlobalEnd(DA, Vec, InsertMode, Vec);
PetscErrorCode DAGlobalToNaturalAllCreate(DA, VecScatter *);
PetscErrorCode DASetUniformCoordinates(DA, PetscReal, PetscReal, PetscReal, PetscReal,
                                       PetscReal, PetscReal);
PetscErrorCode DAGetCoordinateDA(DA, DA *);
PetscErrorCode DAGetCoordinates(DA, Vec *);
PetscErrorCode DAGetGhostedCoordinates(DA, Vec *);
PetscErrorCode DAGetGlobalIndices(DA, PetscInt *, PetscInt **);
PetscErrorCode DAGetAO(DA, AO *);
PetscErrorCode DAGetMatrix(DA, MatType, Mat *);
PetscErrorCode DAGetInterpolation(DA, DA, Mat *, Vec *);

/* ---------------------------------------------------------------- Vec */
PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt, Vec *);
PetscErrorCode VecCreateMPI(MPI_Comm, PetscInt, PetscInt, Vec *);
PetscErrorCode VecCreate(MPI_Comm, Vec *);
PetscErrorCode VecSetSizes(Vec, PetscInt, PetscInt);
PetscErrorCode VecSetFromOptions(Vec);
PetscErrorCode VecDuplicate(Vec, Vec *);
PetscErrorCode VecDestroy(Vec);
PetscErrorCode VecSet(Vec, PetscScalar);
PetscErrorCode VecCopy(Vec, Vec);
PetscErrorCode VecAXPY(Vec, PetscScalar, Vec);
PetscErrorCode VecAYPX(Vec, PetscScalar, Vec);
PetscErrorCode VecWAXPY(Vec, PetscScalar, Vec, Vec);
PetscErrorCode VecAXPBY(Vec, PetscScalar, PetscScalar, Vec);
PetscErrorCode VecScale(Vec, PetscScalar);
PetscErrorCode VecShift(Vec, PetscScalar);
PetscErrorCode VecSum(Vec, PetscScalar *);
PetscErrorCode VecMax(Vec, PetscInt *, PetscReal *);
PetscErrorCode VecMin(Vec, PetscInt *, PetscReal *);
PetscErrorCode VecNorm(Vec, NormType, PetscReal *);
PetscErrorCode VecDot(Vec, Vec, PetscScalar *);
PetscErrorCode VecPointwiseDivide(Vec, Vec, Vec);
PetscErrorCode VecPointwiseMult(Vec, Vec, Vec);
PetscErrorCode VecGetSize(Vec, PetscInt *);
PetscErrorCode VecGetLocalSize(Vec, PetscInt *);
PetscErrorCode VecGetOwnershipRange(Vec, PetscInt *, PetscInt *);
PetscErrorCode VecGetArray(Vec, PetscScalar **);
PetscErrorCode VecRestoreArray(Vec, PetscScalar **);
PetscErrorCode VecGetArray3d(Vec, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt,
                             PetscScalar ****);
PetscErrorCode VecRestoreArray3d(Vec, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt,
                                 PetscInt, PetscScalar ****);
PetscErrorCode VecSetValue(Vec, PetscInt, PetscScalar, InsertMode);
PetscErrorCode VecSetValues(Vec, PetscInt, const PetscInt *, const PetscScalar *, InsertMode);
PetscErrorCode VecGetValues(Vec, PetscInt, const PetscInt *, PetscScalar *);
PetscErrorCode VecAssemblyBegin(Vec);
PetscErrorCode VecAssemblyEnd(Vec);
PetscErrorCode VecView(Vec, PetscViewer);
PetscErrorCode VecLoadIntoVector(PetscViewer, Vec);
PetscErrorCode VecScatterCreateToAll(Vec, VecScatter *, Vec *);
PetscErrorCode VecScatterCreateToZero(Vec, VecScatter *, Vec *);
PetscErrorCode VecScatterBegin(VecScatter, Vec, Vec, InsertMode, ScatterMode);
PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode);
PetscErrorCode VecScatterDestroy(VecScatter);
PetscErrorCode VecStrideScatter(Vec, PetscInt, Vec, InsertMode);

/* ---------------------------------------------------------------- Mat */
PetscErrorCode MatCreate(MPI_Comm, Mat *);
PetscErrorCode MatSetSizes(Mat, PetscInt, PetscInt, PetscInt, PetscInt);
PetscErrorCode MatSetType(Mat, MatType);
PetscErrorCode MatSetFromOptions(Mat);
PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt *, PetscInt,
                                         const PetscInt *);
PetscErrorCode MatSeqAIJSetPreallocation(Mat, PetscInt, const PetscInt *);
PetscErrorCode MatCreateSeqAIJ(MPI_Comm, PetscInt, PetscInt, PetscInt, const PetscInt *, Mat *);
PetscErrorCode MatCreateMPIAIJ(MPI_Comm, PetscInt, PetscInt, PetscInt, PetscInt, PetscInt,
                               const PetscInt *, PetscInt, const PetscInt *, Mat *);
PetscErrorCode MatZeroEntries(Mat);
PetscErrorCode MatSetValues(Mat, PetscInt, const PetscInt *, PetscInt, const PetscInt *,
                            const PetscScalar *, InsertMode);
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType);
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType);
PetscErrorCode MatMult(Mat, Vec, Vec);
PetscErrorCode MatMultAdd(Mat, Vec, Vec, Vec);
PetscErrorCode MatDestroy(Mat);
PetscErrorCode MatGetOwnershipRange(Mat, PetscInt *, PetscInt *);
PetscErrorCode MatGetRow(Mat, PetscInt, PetscInt *, const PetscInt **, const PetscScalar **);
PetscErrorCode MatRestoreRow(Mat, PetscInt, PetscInt *, const PetscInt **, const PetscScalar **);
PetscErrorCode MatCreateShell(MPI_Comm, PetscInt, PetscInt, PetscInt, PetscInt, void *, Mat *);
PetscErrorCode MatShellSetOperation(Mat, MatOperation, void (*)(void));
PetscErrorCode MatShellGetContext(Mat, void *);
PetscErrorCode MatGetVecs(Mat, Vec *, Vec *);
PetscErrorCode MatNullSpaceCreate(MPI_Comm, PetscTruth, PetscInt, const Vec *, MatNullSpace *);
PetscErrorCode MatNullSpaceDestroy(MatNullSpace);
PetscErrorCode MatNullSpaceRemove(MatNullSpace, Vec, Vec *);
PetscErrorCode MatNullSpaceSetFunction(MatNullSpace, PetscErrorCode (*)(Vec, void *), void *);
PetscErrorCode MatCreateSNESMF(SNES, Mat *);
PetscErrorCode MatMFFDComputeJacobian(SNES, Vec, Mat *, Mat *, MatStructure *, void *);
PetscErrorCode MatView(Mat, PetscViewer);

/* ---------------------------------------------------------------- KSP / PC / SNES (inert) */
#define SHIM_INERT(...) (0)
static inline PetscErrorCode KSPCreate(MPI_Comm, KSP *k) { *k = 0; return 0; }
#define KSPDestroy(...) SHIM_INERT()
#define KSPSetType(...) SHIM_INERT()
#define KSPGetPC(...) SHIM_INERT()
#define KSPSetUp(...) SHIM_INERT()
#define KSPSetTolerances(...) SHIM_INERT()
#define KSPSolve(...) SHIM_INERT()
#define KSPSetOperators(...) SHIM_INERT()
#define KSPGMRESSetRestart(...) SHIM_INERT()
#define KSPSetInitialGuessNonzero(...) SHIM_INERT()
#define KSPSetNullSpace(...) SHIM_INERT()
#define KSPSetFromOptions(...) SHIM_INERT()
#define KSPMonitorSet(...) SHIM_INERT()
#define KSPBuildResidual(...) SHIM_INERT()
#define KSPSetNormType(...) SHIM_INERT()
#define KSPSetInitialGuessKnoll(...) SHIM_INERT()
#define KSPGMRESSetPreAllocateVectors(...) SHIM_INERT()
#define KSPAppendOptionsPrefix(...) SHIM_INERT()
#define KSPSetOptionsPrefix(...) SHIM_INERT()
static inline PetscErrorCode KSPMonitorTrueResidualNorm(KSP, PetscInt, PetscReal, void *) { return 0; }
#define KSPMonitorDefault 0
#define KSPGetIterationNumber(k, n) (*(n) = 0, 0)
#define KSPGetResidualNorm(k, r) (*(r) = 0.0, 0)
#define KSPGetConvergedReason(k, r) (0)
#define KSPSetConvergenceTest(...) SHIM_INERT()
#define KSPView(...) SHIM_INERT()
#define PCSetType(...) SHIM_INERT()
#define PCSetUp(...) SHIM_INERT()
#define PCSetOperators(...) SHIM_INERT()
#define PCSetFromOptions(...) SHIM_INERT()
#define PCDestroy(...) SHIM_INERT()
#define PCFactorSetShiftNonzero(...) SHIM_INERT()
#define PCFactorSetShiftType(...) SHIM_INERT()
#define PCFactorSetShiftAmount(...) SHIM_INERT()
#define PCFactorSetLevels(...) SHIM_INERT()
#define PCBJacobiGetSubKSP(...) SHIM_INERT()
#define PCHYPRESetType(...) SHIM_INERT()
#define PCMGSetType(...) SHIM_INERT()
#define PCMGSetLevels(...) SHIM_INERT()
#define PCMGSetCycleType(...) SHIM_INERT()
#define PCMGSetCycles(...) SHIM_INERT()
#define PCMGSetRhs(...) SHIM_INERT()
#define PCMGSetX(...) SHIM_INERT()
#define PCMGSetR(...) SHIM_INERT()
#define PCMGSetRestriction(...) SHIM_INERT()
#define PCMGSetInterpolation(...) SHIM_INERT()
#define PCMGSetResidual(...) SHIM_INERT()
#define PCMGGetSmoother(...) SHIM_INERT()
#define PCMGGetSmootherUp(...) SHIM_INERT()
#define PCMGGetSmootherDown(...) SHIM_INERT()
#define PCMGGetCoarseSolve(...) SHIM_INERT()
#define PCMGSetNumberSmoothUp(...) SHIM_INERT()
#define PCMGSetNumberSmoothDown(...) SHIM_INERT()
#define PCMGDefaultResidual 0
#define PCShellSetApply(...) SHIM_INERT()
#define PCShellSetContext(...) SHIM_INERT()
#define SNESCreate(...) SHIM_INERT()
#define SNESSetType(...) SHIM_INERT()
#define SNESSetFunction(...) SHIM_INERT()
#define SNESSetJacobian(...) SHIM_INERT()
#define SNESSolve(...) SHIM_INERT()
#define SNESSetTolerances(...) SHIM_INERT()
#define SNESGetKSP(...) SHIM_INERT()
#define SNESMonitorSet(...) SHIM_INERT()
#define SNESSetMaxNonlinearStepFailures(...) SHIM_INERT()
#define SNESSetMaxLinearSolveFailures(...) SHIM_INERT()
#define SNESKSPSetUseEW(...) SHIM_INERT()
#define SNESKSPSetParametersEW(...) SHIM_INERT()
#define SNESGetFunctionNorm(s, n) (*(n) = 0.0, 0)
#define SNESDestroy(...) SHIM_INERT()
#define SNESSetFromOptions(...) SHIM_INERT()
#define SNESGetIterationNumber(s, n) (*(n) = 0, 0)
#define SNESGetConvergedReason(...) SHIM_INERT()
#define SNESSetLineSearch(...) SHIM_INERT()
#define SNESDefaultComputeJacobian 0
#define AODestroy(...) SHIM_INERT()
#define AOApplicationToPetsc(...) SHIM_INERT()
#define AOPetscToApplication(...) SHIM_INERT()
#define ISCreateGeneral(...) SHIM_INERT()
#define ISDestroy(...) SHIM_INERT()

/* ---------------------------------------------------------------- misc */
PetscErrorCode PetscInitialize(int *, char ***, const char *, const char *);
PetscErrorCode PetscFinalize(void);
PetscErrorCode PetscPrintf(MPI_Comm, const char *, ...);
PetscErrorCode PetscFPrintf(MPI_Comm, FILE *, const char *, ...);
PetscErrorCode PetscSynchronizedPrintf(MPI_Comm, const char *, ...);
PetscErrorCode PetscSynchronizedFlush(MPI_Comm);
PetscErrorCode PetscGetTime(PetscLogDouble *);
PetscErrorCode PetscBarrier(void *);
PetscErrorCode PetscGlobalSum(const PetscReal *, PetscReal *, MPI_Comm);
PetscErrorCode PetscGlobalMax(const PetscReal *, PetscReal *, MPI_Comm);
PetscErrorCode PetscGlobalMin(const PetscReal *, PetscReal *, MPI_Comm);
PetscErrorCode PetscOptionsGetInt(const char *, const char *, PetscInt *, PetscTruth *);
PetscErrorCode PetscOptionsGetReal(const char *, const char *, PetscReal *, PetscTruth *);
PetscErrorCode PetscOptionsGetTruth(const char *, const char *, PetscTruth *, PetscTruth *);
PetscErrorCode PetscOptionsGetString(const char *, const char *, char *, size_t, PetscTruth *);
PetscErrorCode PetscOptionsGetIntArray(const char *, const char *, PetscInt *, PetscInt *,
                                       PetscTruth *);
PetscErrorCode PetscOptionsGetRealArray(const char *, const char *, PetscReal *, PetscInt *,
                                        PetscTruth *);
PetscErrorCode PetscOptionsHasName(const char *, const char *, PetscTruth *);
PetscErrorCode PetscOptionsInsertString(const char *);
PetscErrorCode PetscOptionsInsertFile(MPI_Comm, const char *, PetscTruth);
PetscErrorCode PetscOptionsClearValue(const char *);
PetscErrorCode PetscOptionsSetValue(const char *, const char *);
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm, const char *, PetscFileMode, PetscViewer *);
PetscErrorCode PetscViewerDestroy(PetscViewer);
#define PetscMalloc(sz, ptr) ((*(void **)(ptr) = calloc(1, (size_t)(sz) + 16)) ? 0 : 1)
#define PetscFree(ptr) (free((void *)(ptr)), 0)
#define PetscMemzero(p, n) (memset((p), 0, (n)), 0)
#define PetscMemcpy(a, b, n) (memcpy((a), (b), (n)), 0)

/* ---------------------------------------------------------------- HYPRE (inert) */
typedef void *HYPRE_Solver;
typedef void *HYPRE_IJMatrix;
typedef void *HYPRE_ParCSRMatrix;
typedef void *HYPRE_IJVector;
typedef void *HYPRE_ParVector;
typedef void *HYPRE_StructGrid;
typedef void *HYPRE_StructStencil;
typedef void *HYPRE_StructMatrix;
typedef void *HYPRE_StructVector;
typedef void *HYPRE_StructSolver;
typedef void *HYPRE_Matrix;
typedef void *HYPRE_Vector;
typedef int (*HYPRE_PtrToSolverFcn)(HYPRE_Solver, HYPRE_Matrix, HYPRE_Vector, HYPRE_Vector);
#define HYPRE_PARCSR 5555
#define HYPRE_BoomerAMGCreate(...) SHIM_INERT()
#define HYPRE_BoomerAMGDestroy(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetup 0
#define HYPRE_BoomerAMGSolve 0
#define HYPRE_BoomerAMGSetInterpType(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetAggNumLevels(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetStrongThreshold(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetTol(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetPrintLevel(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetCoarsenType(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetCycleType(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetMaxIter(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetRelaxType(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetNumSweeps(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetMaxLevels(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetPMaxElmts(...) SHIM_INERT()
#define HYPRE_BoomerAMGSetTruncFactor(...) SHIM_INERT()
#define HYPRE_ParCSRGMRESCreate(...) SHIM_INERT()
#define HYPRE_ParCSRGMRESDestroy(...) SHIM_INERT()
#define HYPRE_ParCSRGMRESSetKDim(...) SHIM_INERT()
#define HYPRE_ParCSRGMRESSetup(...) SHIM_INERT()
#define HYPRE_ParCSRGMRESSolve(...) SHIM_INERT()
#define HYPRE_ParCSRPCGCreate(...) SHIM_INERT()
#define HYPRE_ParCSRPCGDestroy(...) SHIM_INERT()
#define HYPRE_ParCSRPCGSetup(...) SHIM_INERT()
#define HYPRE_ParCSRPCGSolve(...) SHIM_INERT()
#define HYPRE_GMRESSetPrecond(...) SHIM_INERT()
#define HYPRE_GMRESSetMaxIter(...) SHIM_INERT()
#define HYPRE_GMRESSetTol(...) SHIM_INERT()
#define HYPRE_GMRESSetPrintLevel(...) SHIM_INERT()
#define HYPRE_GMRESGetNumIterations(...) SHIM_INERT()
#define HYPRE_GMRESGetFinalRelativeResidualNorm(...) SHIM_INERT()
#define HYPRE_PCGSetPrecond(...) SHIM_INERT()
#define HYPRE_PCGSetMaxIter(...) SHIM_INERT()
#define HYPRE_PCGSetTol(...) SHIM_INERT()
#define HYPRE_PCGSetPrintLevel(...) SHIM_INERT()
#define HYPRE_IJMatrixCreate(...) SHIM_INERT()
#define HYPRE_IJMatrixDestroy(...) SHIM_INERT()
#define HYPRE_IJMatrixSetObjectType(...) SHIM_INERT()
#define HYPRE_IJMatrixInitialize(...) SHIM_INERT()
#define HYPRE_IJMatrixSetValues(...) SHIM_INERT()
#define HYPRE_IJMatrixAddToValues(...) SHIM_INERT()
#define HYPRE_IJMatrixAssemble(...) SHIM_INERT()
#define HYPRE_IJMatrixGetObject(...) SHIM_INERT()
#define HYPRE_IJMatrixSetRowSizes(...) SHIM_INERT()
/* IJ vectors are real (a dense array over [lower, upper]) so that the reference's own
 * right-hand-side assembly and null-space shifts (poisson_hypre.c) run in the oracle. */
int HYPRE_IJVectorCreate(MPI_Comm, int lower, int upper, HYPRE_IJVector *v);
int HYPRE_IJVectorDestroy(HYPRE_IJVector v);
int HYPRE_IJVectorSetObjectType(HYPRE_IJVector v, int t);
int HYPRE_IJVectorInitialize(HYPRE_IJVector v);
int HYPRE_IJVectorSetValues(HYPRE_IJVector v, int n, const int *idx, const double *vals);
int HYPRE_IJVectorAddToValues(HYPRE_IJVector v, int n, const int *idx, const double *vals);
int HYPRE_IJVectorGetValues(HYPRE_IJVector v, int n, const int *idx, double *vals);
int HYPRE_IJVectorAssemble(HYPRE_IJVector v);
int HYPRE_IJVectorGetObject(HYPRE_IJVector v, void **o);
#ifdef __cplusplus
extern "C" {
#endif
double *shim_ij_data(HYPRE_IJVector v, int *n);
#ifdef __cplusplus
}
#endif
#define HYPRE_IJMatrixSetMaxOffProcElmts(...) SHIM_INERT()
#define HYPRE_IJVectorSetMaxOffProcElmts(...) SHIM_INERT()

/* ---------------------------------------------------------------- shim-only helpers */
#ifdef __cplusplus
extern "C" {
#endif
/* CSR export of a recorded matrix: returns nnz; fills row_ptr (m+1), col, val when non-null. */
long shim_mat_to_csr(Mat A, int *row_ptr, int *col, double *val, int *m_out);
#ifdef __cplusplus
}
#endif

#endif /* VFS_PETSC_SHIM_H */
