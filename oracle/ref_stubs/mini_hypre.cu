// Minimal implementation of the HYPRE API subset declared in hypre_stub.h.
// TEST INFRASTRUCTURE ONLY: lets the reference's own generic_simple_v1 (compiled from its source
// tree by oracle/build_ref.sh) run end to end in this repository's test build.  Matrices and
// vectors follow HYPRE's IJ -> ParCSR flow (host set-up, device migration, device data pointers
// that the reference writes into directly); the solves copy the device data to the host and
// run Jacobi-preconditioned CG (PCG) or right-Jacobi BiCGSTAB to
// ||r||_2 <= max(abs_tol, rel_tol * ||b||_2), returning 256 when the iteration cap is hit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <mpi.h>
extern "C" {
#include "hypre_stub.h"
}

struct hypre_IJMatrix_s {
  int n = 0;
  std::vector<int> rowSizes;
  hypre_ParCSRMatrix par{};
  hypre_CSRMatrix diag{}, offd{};
  std::vector<int> I, J;
  std::vector<double> hdata;
  double* ddata = nullptr;
};
struct hypre_IJVector_s {
  int n = 0;
  hypre_ParVector par{};
  hypre_Vector local{};
  std::vector<double> h;
  double* d = nullptr;
  bool onDevice = false;
};
struct hypre_Solver_s {
  bool pcg = true;
  double rtol = 0.0, atol = 0.0;
  int maxit = 1000;
  int its = 0;
  double rel = 0.0;
};

namespace {
void ck(cudaError_t e) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "mini_hypre CUDA error: %s\n", cudaGetErrorString(e));
    std::exit(3);
  }
}
struct HostSys {
  int n;
  const std::vector<int>* I;
  const std::vector<int>* J;
  std::vector<double> a, b, x;
};
HostSys fetch(HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x) {
  hypre_IJMatrix_s* M = static_cast<hypre_IJMatrix_s*>(A->owner);
  HostSys s;
  s.n = M->n;
  s.I = &M->I;
  s.J = &M->J;
  s.a.resize(M->J.size());
  s.b.resize(s.n);
  s.x.resize(s.n);
  ck(cudaDeviceSynchronize());
  ck(cudaMemcpy(s.a.data(), M->diag.data, sizeof(double) * s.a.size(), cudaMemcpyDefault));
  ck(cudaMemcpy(s.b.data(), b->local_vector->data, sizeof(double) * s.n, cudaMemcpyDefault));
  ck(cudaMemcpy(s.x.data(), x->local_vector->data, sizeof(double) * s.n, cudaMemcpyDefault));
  return s;
}
void spmv(const HostSys& s, const std::vector<double>& x, std::vector<double>& y) {
  for (int r = 0; r < s.n; ++r) {
    double acc = 0.0;
    for (int k = (*s.I)[r]; k < (*s.I)[r + 1]; ++k) acc += s.a[k] * x[(*s.J)[k]];
    y[r] = acc;
  }
}
double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}
std::vector<double> dinv(const HostSys& s) {
  std::vector<double> d(s.n, 1.0);
  for (int r = 0; r < s.n; ++r)
    for (int k = (*s.I)[r]; k < (*s.I)[r + 1]; ++k)
      if ((*s.J)[k] == r && s.a[k] != 0.0) d[r] = 1.0 / s.a[k];
  return d;
}
}  // namespace

extern "C" {
HYPRE_Int HYPRE_Initialize(void) { return 0; }
HYPRE_Int HYPRE_Finalize(void) { return 0; }
HYPRE_Int HYPRE_SetMemoryLocation(HYPRE_MemoryLocation) { return 0; }
HYPRE_Int HYPRE_SetExecutionPolicy(HYPRE_ExecutionPolicy) { return 0; }
HYPRE_Int HYPRE_ClearAllErrors(void) { return 0; }

HYPRE_Int HYPRE_IJMatrixCreate(MPI_Comm, HYPRE_BigInt il, HYPRE_BigInt iu, HYPRE_BigInt, HYPRE_BigInt, HYPRE_IJMatrix* A) {
  *A = new hypre_IJMatrix_s();
  (*A)->n = (int)(iu - il + 1);
  return 0;
}
HYPRE_Int HYPRE_IJMatrixSetObjectType(HYPRE_IJMatrix, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_IJMatrixSetRowSizes(HYPRE_IJMatrix A, const HYPRE_Int* s) {
  A->rowSizes.assign(s, s + A->n);
  return 0;
}
HYPRE_Int HYPRE_IJMatrixInitialize_v2(HYPRE_IJMatrix, HYPRE_MemoryLocation) { return 0; }
HYPRE_Int HYPRE_IJMatrixInitialize(HYPRE_IJMatrix) { return 0; }
HYPRE_Int HYPRE_IJMatrixSetValues(HYPRE_IJMatrix A, HYPRE_Int nrows, HYPRE_Int* ncols, const HYPRE_BigInt*,
                                  const HYPRE_BigInt* cols, const HYPRE_Complex* vals) {
  A->I.assign(nrows + 1, 0);
  for (int r = 0; r < nrows; ++r) A->I[r + 1] = A->I[r] + ncols[r];
  A->J.resize(A->I[nrows]);
  A->hdata.resize(A->I[nrows]);
  for (int k = 0; k < A->I[nrows]; ++k) {
    A->J[k] = (int)cols[k];
    A->hdata[k] = vals[k];
  }
  return 0;
}
HYPRE_Int HYPRE_IJMatrixAssemble(HYPRE_IJMatrix A) {
  A->diag.num_rows = A->n;
  A->diag.num_nonzeros = (int)A->J.size();
  A->diag.i = A->I.data();
  A->diag.j = A->J.data();
  A->diag.data = A->ddata ? A->ddata : A->hdata.data();
  A->offd = hypre_CSRMatrix{A->n, 0, nullptr, nullptr, nullptr};
  A->par.diag = &A->diag;
  A->par.offd = &A->offd;
  A->par.owner = A;
  if (A->ddata) ck(cudaMemcpy(A->ddata, A->hdata.data(), sizeof(double) * A->hdata.size(), cudaMemcpyHostToDevice));
  return 0;
}
HYPRE_Int HYPRE_IJMatrixGetObject(HYPRE_IJMatrix A, void** o) {
  *o = &A->par;
  return 0;
}
HYPRE_Int HYPRE_IJMatrixMigrate(HYPRE_IJMatrix A, HYPRE_MemoryLocation loc) {
  if (loc == HYPRE_MEMORY_DEVICE && !A->ddata) {
    ck(cudaMalloc(&A->ddata, sizeof(double) * std::max<size_t>(A->hdata.size(), 1)));
    ck(cudaMemcpy(A->ddata, A->hdata.data(), sizeof(double) * A->hdata.size(), cudaMemcpyHostToDevice));
    A->diag.data = A->ddata;
  }
  return 0;
}
HYPRE_Int HYPRE_IJMatrixDestroy(HYPRE_IJMatrix A) {
  if (A->ddata) cudaFree(A->ddata);
  delete A;
  return 0;
}
HYPRE_Int HYPRE_IJVectorCreate(MPI_Comm, HYPRE_BigInt il, HYPRE_BigInt iu, HYPRE_IJVector* v) {
  *v = new hypre_IJVector_s();
  (*v)->n = (int)(iu - il + 1);
  (*v)->h.assign((*v)->n, 0.0);
  return 0;
}
HYPRE_Int HYPRE_IJVectorSetObjectType(HYPRE_IJVector, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_IJVectorInitialize_v2(HYPRE_IJVector, HYPRE_MemoryLocation) { return 0; }
HYPRE_Int HYPRE_IJVectorInitialize(HYPRE_IJVector) { return 0; }
HYPRE_Int HYPRE_IJVectorSetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt* idx, const HYPRE_Complex* x) {
  for (int k = 0; k < n; ++k) v->h[(size_t)idx[k]] = x[k];
  return 0;
}
HYPRE_Int HYPRE_IJVectorAssemble(HYPRE_IJVector v) {
  v->local.size = v->n;
  v->local.data = v->onDevice ? v->d : v->h.data();
  v->par.local_vector = &v->local;
  return 0;
}
HYPRE_Int HYPRE_IJVectorMigrate(HYPRE_IJVector v, HYPRE_MemoryLocation loc) {
  if (loc == HYPRE_MEMORY_DEVICE && !v->onDevice) {
    if (!v->d) ck(cudaMalloc(&v->d, sizeof(double) * std::max(v->n, 1)));
    ck(cudaMemcpy(v->d, v->h.data(), sizeof(double) * v->n, cudaMemcpyHostToDevice));
    v->onDevice = true;
  } else if (loc == HYPRE_MEMORY_HOST && v->onDevice) {
    ck(cudaDeviceSynchronize());
    ck(cudaMemcpy(v->h.data(), v->d, sizeof(double) * v->n, cudaMemcpyDeviceToHost));
    v->onDevice = false;
  }
  v->local.data = v->onDevice ? v->d : v->h.data();
  return 0;
}
HYPRE_Int HYPRE_IJVectorGetObject(HYPRE_IJVector v, void** o) {
  *o = &v->par;
  return 0;
}
HYPRE_Int HYPRE_IJVectorGetValues(HYPRE_IJVector v, HYPRE_Int n, const HYPRE_BigInt* idx, HYPRE_Complex* x) {
  for (int k = 0; k < n; ++k) x[k] = v->h[(size_t)idx[k]];
  return 0;
}
HYPRE_Int HYPRE_IJVectorDestroy(HYPRE_IJVector v) {
  if (v->d) cudaFree(v->d);
  delete v;
  return 0;
}

HYPRE_Int anb_stub_new_solver(HYPRE_Solver* s, bool pcg) {
  *s = new hypre_Solver_s();
  (*s)->pcg = pcg;
  return 0;
}
HYPRE_Int HYPRE_ParCSRPCGCreate(MPI_Comm, HYPRE_Solver* s) { return anb_stub_new_solver(s, true); }
HYPRE_Int HYPRE_ParCSRPCGDestroy(HYPRE_Solver s) { delete s; return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetTol(HYPRE_Solver s, HYPRE_Real t) { s->rtol = t; return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetAbsoluteTol(HYPRE_Solver s, HYPRE_Real t) { s->atol = t; return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetMaxIter(HYPRE_Solver s, HYPRE_Int m) { s->maxit = m; return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetTwoNorm(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetPrintLevel(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetLogging(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetPrecond(HYPRE_Solver, HYPRE_PtrToParSolverFcn, HYPRE_PtrToParSolverFcn, HYPRE_Solver) { return 0; }
HYPRE_Int HYPRE_ParCSRPCGSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { return 0; }
HYPRE_Int HYPRE_ParCSRPCGSolve(HYPRE_Solver sv, HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x) {
  HostSys s = fetch(A, b, x);
  const int n = s.n;
  std::vector<double> d = dinv(s), r(n), z(n), p(n), q(n);
  spmv(s, s.x, r);
  for (int i = 0; i < n; ++i) r[i] = s.b[i] - r[i];
  const double bn = std::sqrt(dot(s.b, s.b));
  const double eps = std::max(sv->atol, sv->rtol * bn);
  double rr = dot(r, r);
  int it = 0;
  HYPRE_Int rc = 0;
  if (std::sqrt(rr) > eps) {
    for (int i = 0; i < n; ++i) { z[i] = d[i] * r[i]; p[i] = z[i]; }
    double rz = dot(r, z);
    while (true) {
      if (it >= sv->maxit) { rc = 256; break; }
      ++it;
      spmv(s, p, q);
      const double al = rz / dot(p, q);
      for (int i = 0; i < n; ++i) { s.x[i] += al * p[i]; r[i] -= al * q[i]; }
      rr = dot(r, r);
      if (std::sqrt(rr) <= eps) break;
      for (int i = 0; i < n; ++i) z[i] = d[i] * r[i];
      const double rzn = dot(r, z);
      const double be = rzn / rz;
      rz = rzn;
      for (int i = 0; i < n; ++i) p[i] = z[i] + be * p[i];
    }
  }
  sv->its = it;
  sv->rel = bn > 0 ? std::sqrt(rr) / bn : 0.0;
  ck(cudaMemcpy(x->local_vector->data, s.x.data(), sizeof(double) * n, cudaMemcpyDefault));
  return rc;
}
HYPRE_Int HYPRE_ParCSRPCGGetNumIterations(HYPRE_Solver s, HYPRE_Int* n) { *n = s->its; return 0; }
HYPRE_Int HYPRE_ParCSRPCGGetFinalRelativeResidualNorm(HYPRE_Solver s, HYPRE_Real* r) { *r = s->rel; return 0; }

HYPRE_Int HYPRE_ParCSRBiCGSTABCreate(MPI_Comm, HYPRE_Solver* s) { return anb_stub_new_solver(s, false); }
HYPRE_Int HYPRE_ParCSRBiCGSTABDestroy(HYPRE_Solver s) { delete s; return 0; }
HYPRE_Int HYPRE_ParCSRBiCGSTABSetTol(HYPRE_Solver s, HYPRE_Real t) { s->rtol = t; return 0; }
HYPRE_Int HYPRE_ParCSRBiCGSTABSetAbsoluteTol(HYPRE_Solver s, HYPRE_Real t) { s->atol = t; return 0; }
HYPRE_Int HYPRE_ParCSRBiCGSTABSetMaxIter(HYPRE_Solver s, HYPRE_Int m) { s->maxit = m; return 0; }
HYPRE_Int HYPRE_ParCSRBiCGSTABSetPrintLevel(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_ParCSRBiCGSTABSetLogging(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_ParCSRBiCGSTABSetPrecond(HYPRE_Solver, HYPRE_PtrToParSolverFcn, HYPRE_PtrToParSolverFcn, HYPRE_Solver) { return 0; }
HYPRE_Int HYPRE_ParCSRBiCGSTABSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { return 0; }
HYPRE_Int HYPRE_ParCSRBiCGSTABSolve(HYPRE_Solver sv, HYPRE_ParCSRMatrix A, HYPRE_ParVector b, HYPRE_ParVector x) {
  HostSys s = fetch(A, b, x);
  const int n = s.n;
  std::vector<double> d = dinv(s), r(n), rh(n), p(n, 0.0), v(n, 0.0), sv2(n), t(n), ph(n), sh(n);
  spmv(s, s.x, r);
  for (int i = 0; i < n; ++i) r[i] = s.b[i] - r[i];
  rh = r;
  const double bn = std::sqrt(dot(s.b, s.b));
  const double eps = std::max(sv->atol, sv->rtol * bn);
  double rn = std::sqrt(dot(r, r));
  double rho = 1.0, al = 1.0, om = 1.0;
  int it = 0;
  HYPRE_Int rc = 0;
  while (rn > eps) {
    if (it >= sv->maxit) { rc = 256; break; }
    ++it;
    const double rhon = dot(rh, r);
    const double be = (rhon / rho) * (al / om);
    rho = rhon;
    for (int i = 0; i < n; ++i) { p[i] = r[i] + be * (p[i] - om * v[i]); ph[i] = d[i] * p[i]; }
    spmv(s, ph, v);
    al = rho / dot(rh, v);
    for (int i = 0; i < n; ++i) sv2[i] = r[i] - al * v[i];
    if (std::sqrt(dot(sv2, sv2)) <= eps) {
      for (int i = 0; i < n; ++i) s.x[i] += al * ph[i];
      rn = std::sqrt(dot(sv2, sv2));
      break;
    }
    for (int i = 0; i < n; ++i) sh[i] = d[i] * sv2[i];
    spmv(s, sh, t);
    const double tt = dot(t, t);
    om = tt > 0 ? dot(t, sv2) / tt : 0.0;
    for (int i = 0; i < n; ++i) { s.x[i] += al * ph[i] + om * sh[i]; r[i] = sv2[i] - om * t[i]; }
    rn = std::sqrt(dot(r, r));
    if (om == 0.0) { rc = 256; break; }
  }
  sv->its = it;
  sv->rel = bn > 0 ? rn / bn : 0.0;
  ck(cudaMemcpy(x->local_vector->data, s.x.data(), sizeof(double) * n, cudaMemcpyDefault));
  return rc;
}
HYPRE_Int HYPRE_ParCSRBiCGSTABGetNumIterations(HYPRE_Solver s, HYPRE_Int* n) { *n = s->its; return 0; }
HYPRE_Int HYPRE_ParCSRBiCGSTABGetFinalRelativeResidualNorm(HYPRE_Solver s, HYPRE_Real* r) { *r = s->rel; return 0; }
HYPRE_Int HYPRE_ParCSRDiagScale(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { return 0; }
HYPRE_Int HYPRE_ParCSRDiagScaleSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { return 0; }
HYPRE_Int HYPRE_BoomerAMGCreate(HYPRE_Solver* s) { return anb_stub_new_solver(s, true); }
HYPRE_Int HYPRE_BoomerAMGDestroy(HYPRE_Solver s) { delete s; return 0; }
HYPRE_Int HYPRE_BoomerAMGSetup(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSolve(HYPRE_Solver, HYPRE_ParCSRMatrix, HYPRE_ParVector, HYPRE_ParVector) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetTol(HYPRE_Solver, HYPRE_Real) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetMaxIter(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetPrintLevel(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetLogging(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetCoarsenType(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetInterpType(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetRelaxType(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetNumSweeps(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetPMaxElmts(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetTruncFactor(HYPRE_Solver, HYPRE_Real) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetKeepTranspose(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetRAP2(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetAggNumLevels(HYPRE_Solver, HYPRE_Int) { return 0; }
HYPRE_Int HYPRE_BoomerAMGSetAggInterpType(HYPRE_Solver, HYPRE_Int) { return 0; }
}
