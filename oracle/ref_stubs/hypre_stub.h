/* Stand-in declarations for the HYPRE 3.0.0 API subset used by the reference's
 * apps/generic_simple_v1/src/main.cu, so that file compiles in this repository's test build.
 * TEST INFRASTRUCTURE ONLY: implemented by mini_hypre.cu with plain Jacobi-preconditioned
 * CG / BiCGSTAB solves on the host (BoomerAMG settings are accepted and ignored). */
#ifndef ANB_HYPRE_STUB_H
#define ANB_HYPRE_STUB_H
#include <mpi.h>
typedef int HYPRE_Int;
typedef long long HYPRE_BigInt;
typedef double HYPRE_Complex;
typedef double HYPRE_Real;
typedef struct hypre_CSRMatrix_s {
  HYPRE_Int num_rows, num_nonzeros;
  HYPRE_Int *i, *j;
  HYPRE_Complex *data;
} hypre_CSRMatrix;
typedef struct hypre_ParCSRMatrix_s {
  hypre_CSRMatrix *diag, *offd;
  void *owner; /* back-pointer to the IJ matrix (stand-in bookkeeping) */
} hypre_ParCSRMatrix;
typedef struct hypre_Vector_s {
  HYPRE_Int size;
  HYPRE_Complex *data;
} hypre_Vector;
typedef struct hypre_ParVector_s {
  hypre_Vector *local_vector;
} hypre_ParVector;
typedef struct hypre_IJMatrix_s *HYPRE_IJMatrix;
typedef struct hypre_IJVector_s *HYPRE_IJVector;
typedef hypre_ParCSRMatrix *HYPRE_ParCSRMatrix;
typedef hypre_ParVector *HYPRE_ParVector;
typedef struct hypre_Solver_s *HYPRE_Solver;
typedef HYPRE_Int (*HYPRE_PtrToParSolverFcn)(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
typedef enum { HYPRE_MEMORY_HOST = 0, HYPRE_MEMORY_DEVICE = 1 } HYPRE_MemoryLocation;
typedef enum { HYPRE_EXEC_HOST = 0, HYPRE_EXEC_DEVICE = 1 } HYPRE_ExecutionPolicy;
#define HYPRE_PARCSR 5555
#define hypre_ParCSRMatrixDiag(m) ((m)->diag)
#define hypre_ParCSRMatrixOffd(m) ((m)->offd)
#define hypre_CSRMatrixI(m) ((m)->i)
#define hypre_CSRMatrixJ(m) ((m)->j)
#define hypre_CSRMatrixData(m) ((m)->data)
#define hypre_CSRMatrixNumNonzeros(m) ((m)->num_nonzeros)
#define hypre_ParVectorLocalVector(v) ((v)->local_vector)
#define hypre_VectorData(v) ((v)->data)
HYPRE_Int HYPRE_Initialize(void);
HYPRE_Int HYPRE_Finalize(void);
HYPRE_Int HYPRE_SetMemoryLocation(HYPRE_MemoryLocation);
HYPRE_Int HYPRE_SetExecutionPolicy(HYPRE_ExecutionPolicy);
HYPRE_Int HYPRE_ClearAllErrors(void);
HYPRE_Int HYPRE_IJMatrixCreate(MPI_Comm, HYPRE_BigInt, HYPRE_BigInt, HYPRE_BigInt, HYPRE_BigInt, HYPRE_IJMatrix*);
HYPRE_Int HYPRE_IJMatrixSetObjectType(HYPRE_IJMatrix, HYPRE_Int);
HYPRE_Int HYPRE_IJMatrixSetRowSizes(HYPRE_IJMatrix, const HYPRE_Int*);
HYPRE_Int HYPRE_IJMatrixInitialize_v2(HYPRE_IJMatrix, HYPRE_MemoryLocation);
HYPRE_Int HYPRE_IJMatrixInitialize(HYPRE_IJMatrix);
HYPRE_Int HYPRE_IJMatrixSetValues(HYPRE_IJMatrix, HYPRE_Int, HYPRE_Int*, const HYPRE_BigInt*, const HYPRE_BigInt*, const HYPRE_Complex*);
HYPRE_Int HYPRE_IJMatrixAssemble(HYPRE_IJMatrix);
HYPRE_Int HYPRE_IJMatrixGetObject(HYPRE_IJMatrix, void**);
HYPRE_Int HYPRE_IJMatrixMigrate(HYPRE_IJMatrix, HYPRE_MemoryLocation);
HYPRE_Int HYPRE_IJMatrixDestroy(HYPRE_IJMatrix);
HYPRE_Int HYPRE_IJVectorCreate(MPI_Comm, HYPRE_BigInt, HYPRE_BigInt, HYPRE_IJVector*);
HYPRE_Int HYPRE_IJVectorSetObjectType(HYPRE_IJVector, HYPRE_Int);
HYPRE_Int HYPRE_IJVectorInitialize_v2(HYPRE_IJVector, HYPRE_MemoryLocation);
HYPRE_Int HYPRE_IJVectorInitialize(HYPRE_IJVector);
HYPRE_Int HYPRE_IJVectorSetValues(HYPRE_IJVector, HYPRE_Int, const HYPRE_BigInt*, const HYPRE_Complex*);
HYPRE_Int HYPRE_IJVectorAssemble(HYPRE_IJVector);
HYPRE_Int HYPRE_IJVectorMigrate(HYPRE_IJVector, HYPRE_MemoryLocation);
HYPRE_Int HYPRE_IJVectorGetObject(HYPRE_IJVector, void**);
HYPRE_Int HYPRE_IJVectorGetValues(HYPRE_IJVector, HYPRE_Int, const HYPRE_BigInt*, HYPRE_Complex*);
HYPRE_Int HYPRE_IJVectorDestroy(HYPRE_IJVector);
HYPRE_Int HYPRE_ParCSRPCGCreate(MPI_Comm, HYPRE_Solver*);
HYPRE_Int HYPRE_ParCSRPCGDestroy(HYPRE_Solver);
HYPRE_Int HYPRE_ParCSRPCGSetTol(HYPRE_Solver, HYPRE_Real);
HYPRE_Int HYPRE_ParCSRPCGSetAbsoluteTol(HYPRE_Solver, HYPRE_Real);
HYPRE_Int HYPRE_ParCSRPCGSetMaxIter(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_ParCSRPCGSetTwoNorm(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_ParCSRPCGSetPrintLevel(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_ParCSRPCGSetLogging(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_ParCSRPCGSetPrecond(HYPRE_Solver, HYPRE_PtrToParSolverFcn, HYPRE_PtrToParSolverFcn, HYPRE_Solver);
HYPRE_Int HYPRE_ParCSRPCGSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_ParCSRPCGSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_ParCSRPCGGetNumIterations(HYPRE_Solver, HYPRE_Int*);
HYPRE_Int HYPRE_ParCSRPCGGetFinalRelativeResidualNorm(HYPRE_Solver, HYPRE_Real*);
HYPRE_Int HYPRE_ParCSRBiCGSTABCreate(MPI_Comm, HYPRE_Solver*);
HYPRE_Int HYPRE_ParCSRBiCGSTABDestroy(HYPRE_Solver);
HYPRE_Int HYPRE_ParCSRBiCGSTABSetTol(HYPRE_Solver, HYPRE_Real);
HYPRE_Int HYPRE_ParCSRBiCGSTABSetAbsoluteTol(HYPRE_Solver, HYPRE_Real);
HYPRE_Int HYPRE_ParCSRBiCGSTABSetMaxIter(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_ParCSRBiCGSTABSetPrintLevel(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_ParCSRBiCGSTABSetLogging(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_ParCSRBiCGSTABSetPrecond(HYPRE_Solver, HYPRE_PtrToParSolverFcn, HYPRE_PtrToParSolverFcn, HYPRE_Solver);
HYPRE_Int HYPRE_ParCSRBiCGSTABSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_ParCSRBiCGSTABSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_ParCSRBiCGSTABGetNumIterations(HYPRE_Solver, HYPRE_Int*);
HYPRE_Int HYPRE_ParCSRBiCGSTABGetFinalRelativeResidualNorm(HYPRE_Solver, HYPRE_Real*);
HYPRE_Int HYPRE_ParCSRDiagScale(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_ParCSRDiagScaleSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_BoomerAMGCreate(HYPRE_Solver*);
HYPRE_Int HYPRE_BoomerAMGDestroy(HYPRE_Solver);
HYPRE_Int HYPRE_BoomerAMGSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_BoomerAMGSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector);
HYPRE_Int HYPRE_BoomerAMGSetTol(HYPRE_Solver, HYPRE_Real);
HYPRE_Int HYPRE_BoomerAMGSetMaxIter(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetPrintLevel(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetLogging(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetCoarsenType(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetInterpType(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetRelaxType(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetNumSweeps(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetPMaxElmts(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetTruncFactor(HYPRE_Solver, HYPRE_Real);
HYPRE_Int HYPRE_BoomerAMGSetKeepTranspose(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetRAP2(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetAggNumLevels(HYPRE_Solver, HYPRE_Int);
HYPRE_Int HYPRE_BoomerAMGSetAggInterpType(HYPRE_Solver, HYPRE_Int);
#endif
