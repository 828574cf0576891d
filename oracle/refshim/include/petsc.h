// Stand-in for the slice of PETSc's C API that the reference's src/Math/SparseMatrix.cpp and
// SparseVector.cpp call, so that its solver sources compile and run here without PETSc.
// Test infrastructure only: matrices are kept row by row with PETSc's insertion rules
// (INSERT_VALUES overwrites, negative row or column indices are ignored); KSPSolve records
// every system it is given and solves it tightly (refshim.cpp), in place of PETSc's
// KSPBCGS + PCSOR.  One process, so every ownership range is the whole object.
#ifndef CAFFE_REFSHIM_PETSC_H
#define CAFFE_REFSHIM_PETSC_H

// the C headers petsc.h brings in with it (petscsys.h / petscmath.h), which the reference relies on
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int PetscErrorCode;
typedef int PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscComm;

typedef struct RefshimMat* Mat;
typedef struct RefshimVec* Vec;
typedef struct RefshimKsp* KSP;
typedef struct RefshimKsp* PC;   // the preconditioner is a property of the solver here
typedef struct RefshimViewer* PetscViewer;

typedef const char* MatType;
typedef const char* VecType;
typedef const char* KSPType;
typedef const char* PCType;

#define PETSC_COMM_WORLD 0
#define PETSC_DECIDE (-1)
#define PETSC_DEFAULT (-2)
#define PETSC_NULL nullptr
#define MATAIJ "aij"
#define VECSTANDARD "standard"
#define KSPBCGS "bcgs"
#define PCSOR "sor"
#define PETSC_VIEWER_STDOUT_SELF ((PetscViewer)0)

typedef enum { NOT_SET_VALUES, INSERT_VALUES, ADD_VALUES } InsertMode;
typedef enum { MAT_FINAL_ASSEMBLY = 0, MAT_FLUSH_ASSEMBLY = 1 } MatAssemblyType;
typedef enum { NORM_1 = 0, NORM_2 = 1, NORM_FROBENIUS = 2, NORM_INFINITY = 3 } NormType;
typedef enum { MAT_INITIAL_MATRIX, MAT_REUSE_MATRIX } MatReuse;

PetscErrorCode PetscInitializeNoArguments(void);

PetscErrorCode MatCreate(PetscComm, Mat*);
PetscErrorCode MatSetSizes(Mat, PetscInt m, PetscInt n, PetscInt M, PetscInt N);
PetscErrorCode MatSetType(Mat, MatType);
PetscErrorCode MatMPIAIJSetPreallocation(Mat, PetscInt, const PetscInt*, PetscInt, const PetscInt*);
PetscErrorCode MatSeqAIJSetPreallocation(Mat, PetscInt, const PetscInt*);
PetscErrorCode MatSetUp(Mat);
PetscErrorCode MatGetOwnershipRange(Mat, PetscInt*, PetscInt*);
PetscErrorCode MatDestroy(Mat*);
PetscErrorCode MatSetValues(Mat, PetscInt nr, const PetscInt* rows, PetscInt nc, const PetscInt* cols, const PetscScalar* v,
                            InsertMode);
PetscErrorCode MatZeroEntries(Mat);
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType);
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType);
PetscErrorCode MatView(Mat, PetscViewer);
PetscErrorCode MatMatMult(Mat, Mat, MatReuse, PetscReal, Mat*);
PetscErrorCode MatMult(Mat, Vec, Vec);
PetscErrorCode MatMultAdd(Mat, Vec, Vec, Vec);
PetscErrorCode MatScale(Mat, PetscScalar);

PetscErrorCode KSPCreate(PetscComm, KSP*);
PetscErrorCode KSPDestroy(KSP*);
PetscErrorCode KSPSetOperators(KSP, Mat, Mat);
PetscErrorCode KSPGetPC(KSP, PC*);
PetscErrorCode PCSetType(PC, PCType);
PetscErrorCode PCSORSetIterations(PC, PetscInt, PetscInt);
PetscErrorCode KSPSetTolerances(KSP, PetscReal rtol, PetscReal abstol, PetscReal dtol, PetscInt maxits);
PetscErrorCode KSPSetType(KSP, KSPType);
PetscErrorCode KSPSolve(KSP, Vec b, Vec x);
PetscErrorCode KSPGetIterationNumber(KSP, PetscInt*);

PetscErrorCode PetscViewerASCIIOpen(PetscComm, const char*, PetscViewer*);
PetscErrorCode PetscViewerDestroy(PetscViewer*);

PetscErrorCode VecCreate(PetscComm, Vec*);
PetscErrorCode VecSetSizes(Vec, PetscInt n, PetscInt N);
PetscErrorCode VecSetType(Vec, VecType);
PetscErrorCode VecGetOwnershipRange(Vec, PetscInt*, PetscInt*);
PetscErrorCode VecDuplicate(Vec, Vec*);
PetscErrorCode VecDestroy(Vec*);
PetscErrorCode VecSetValues(Vec, PetscInt n, const PetscInt* ix, const PetscScalar* y, InsertMode);
PetscErrorCode VecZeroEntries(Vec);
PetscErrorCode VecGetValues(Vec, PetscInt n, const PetscInt* ix, PetscScalar* y);
PetscErrorCode VecNorm(Vec, NormType, PetscReal*);
PetscErrorCode VecView(Vec, PetscViewer);
PetscErrorCode VecScale(Vec, PetscScalar);
PetscErrorCode VecAssemblyBegin(Vec);
PetscErrorCode VecAssemblyEnd(Vec);

#endif
