// Launch wrappers for the SIMPLE kernels (implemented in kernels.cu).
#pragma once

#include "device.cuh"

#include <atomic>
#include <vector>

namespace anb {

// Kernel families that can be timed with CUDA events (anb_profile_select in include/anb.h).
enum KernelFamily {
  kKfNone = 0, kKfGradient = 1, kKfMomentum = 2, kKfPressureRc = 3, kKfNonOrth = 4, kKfFluxFinal = 5,
  kKfBicgSpmv = 6, kKfPcgSpmv = 7, kKfAmgResid0 = 8, kKfAmgUp0 = 9, kKfAmgCoarse = 10, kKfPcgUpdate = 11,
  kKfBicgVector = 12, kKfCount = 13
};

// Event-pair recorder for one selected kernel family on one stream.
struct Prof {
  int family = kKfNone;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  long long launches = 0;
  double seconds = 0.0, bytes = 0.0;
  cudaEvent_t next() {
    if (used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[used++];
  }
  // call after the stream is synchronized
  void flush() {
    for (size_t k = 0; k + 1 < used; k += 2) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, pool[k], pool[k + 1]) == cudaSuccess) seconds += ms * 1e-3;
    }
    used = 0;
  }
  ~Prof() {
    for (auto e : pool) cudaEventDestroy(e);
  }
};

extern std::atomic<long long> g_launches;

struct AlgoBytes;
struct LaunchCfg {
  int rowBlocks;   // grid for row-parallel kernels (grid-stride)
  cudaStream_t stream;
  Prof* prof = nullptr;
  const AlgoBytes* ab = nullptr;
};

// Records a start/stop event pair around the launches in its scope when `fam` is selected.
struct ProfScope {
  const LaunchCfg& lc;
  bool on;
  ProfScope(const LaunchCfg& l, int fam, double bytes, int nLaunch = 1) : lc(l) {
    g_launches += nLaunch;
    on = lc.prof && lc.prof->family == fam;
    if (on) {
      cudaEventRecord(lc.prof->next(), lc.stream);
      lc.prof->launches += 1;
      lc.prof->bytes += bytes;
    }
  }
  ~ProfScope() {
    if (on) cudaEventRecord(lc.prof->next(), lc.stream);
  }
};

// Algorithmic (compulsory) bytes of one launch, used for the roofline report.
struct AlgoBytes {
  double gradient(int nf) const;
  double momentum() const;
  double pressure_rc() const;
  double nonorth() const;
  double flux_final() const;
  double bicg_spmv(int nc) const;
  double pcg_spmv() const;
  int C = 0, Fi = 0, Fb = 0;
  long long nnzOff = 0;
};

// Least-squares gradients of up to four cell fields.  fieldBit selects the Dirichlet bit in
// DMesh::bType (1 u, 2 v, 4 w, 8 p); bval the matching boundary values.  g[f] -> 3*nCells SoA.
struct GradArgs {
  int nf;
  const double* phi[4];
  unsigned char bit[4];
  const double* bval[4];
  double* g[4];
};
void launch_lsq_grad(const LaunchCfg& lc, const DMesh& m, const GradArgs& a);

struct MomArgs {
  const double* U;    // 3*nCells old velocity (convecting velocity)
  const double* Q;    // 3*nCells field of the relaxation term (old field, or current iterate)
  const double* G;    // gradients of Q: [grad q0 | grad q1 | grad q2 | grad p], each 3*nCells SoA
  double rho, mu, uRelax;
  int relax;
  int rhsOnly;        // 1: right-hand sides only, relaxation from the stored relaxed diagonal
  double* val;
  double* diag;
  double* rhs;        // 3*nCells
  double* rau;
};
void launch_momentum(const LaunchCfg& lc, const DMesh& m, const MomArgs& a);

struct PresArgs {
  const double* Us;   // 3*nCells momentum solution
  const double* P;
  const double* Gp;   // 3*nCells SoA
  const double* rau;
  double rho;
  double* val;
  double* diag;
  double* phiStar;    // nInternal + nBoundary
  double* divStar;
  double* b;          // first pressure right-hand side, -divStar
  double* pc;         // zeroed p'
  double* wdinv;      // optional: omega / diag for the AMG smoother
  double omega;
};
void launch_pressure_rc(const LaunchCfg& lc, const DMesh& m, const PresArgs& a);

struct NonOrthArgs {
  const double* rau;
  const double* Gc;   // grad p' (3*nCells SoA)
  const double* divBase;
  double* b;
};
void launch_nonorth_rhs(const LaunchCfg& lc, const DMesh& m, const NonOrthArgs& a);

struct FluxArgs {
  const double* rau;
  const double* Gc;
  const double* pc;
  const double* phiStar;
  double* phi;
  double* divCorr;
  int update;         // 1: also p += pRelax p', U = Us - rAU grad p', and the step statistics
  double pRelax;
  double* P;
  double* U;          // in: old velocity, out: corrected velocity
  const double* Us;
  Reducer red;
  double* stats;      // 9 doubles: sum du^2, u^2, dv^2, v^2, dw^2, w^2, dp^2, p^2, max|div|
};
void launch_flux_final(const LaunchCfg& lc, const DMesh& m, const FluxArgs& a);

// Patch force (compute_patch_forces_wall_shear, main.cu:2828-2933) over boundary faces
// [b0, b1); out: Fp[3] Fv[3] F[3] area nFaces minDn maxDn maxUt maxShear (15 doubles).
void launch_patch_force(cudaStream_t s, const DMesh& m, int b0, int b1, int sign, double mu,
                        const double* bA, const double* bN, const double* U, const double* P, double* out);

// ---- Krylov ----------------------------------------------------------------------------
struct BicgArgs {
  DSell A;
  int nc;             // components (1..3), vectors are nc*n
  const double* b;
  double* x;
  double *r, *rh, *p, *v, *s, *t, *ph, *sh;
  double* sc;         // per component 8 scalars: rho, rhoN, alpha, omega, eps, rn, tsum, ssum
  int* fl;            // per component 4 ints: done, half, iters, converged
  double atol, rtol;
  int maxit;
  Reducer red;
};
void bicg_init(const LaunchCfg& lc, const BicgArgs& a);
void bicg_iteration(const LaunchCfg& lc, const BicgArgs& a);

struct AmgDev;  // hierarchy on the device (amg.cu)

struct PcgArgs {
  DSell A;
  const double* b;
  double* x;
  double *r, *z, *p0, *p1, *q;
  double* sc;         // rz, alpha, beta, eps, rr, pq
  int* fl;            // done, iters, converged, first
  double atol, rtol;
  int maxit;
  Reducer red;
};
void pcg_init(const LaunchCfg& lc, const PcgArgs& a);
// one iteration; `it` selects the p double buffer; precond == nullptr -> Jacobi
void pcg_iteration(const LaunchCfg& lc, const PcgArgs& a, int it, const AmgDev* amg);
// z = M^-1 r for the first iteration (and rz)
void pcg_precondition(const LaunchCfg& lc, const PcgArgs& a, const AmgDev* amg);

// ---- AMG (aggregation, V-cycle) ------------------------------------------------------------
struct AmgLevelDev {
  int n, nc;
  // matrix of this level: level 0 borrows the pressure matrix (SELL-32 slices in sliceOff),
  // coarser levels are CSR (rowOff)
  const int* sliceOff;
  const int* rowOff;
  const int* col;
  double* val;
  double* diag;
  // restriction to the next level
  const int* agg;
  const int* memOff;
  const int* mem;
  const int* gOff;     // Galerkin gather for the next level's storage
  const int* gIdx;
  int nEntNext;        // next level's SELL storage entries
  // work vectors
  double *b, *x, *x2;
  double* wdinv;       // omega / diag (Jacobi smoother)
};
struct AmgDev {
  int nLevels = 0;
  AmgLevelDev lv[24];
  double* dense = nullptr;   // coarsest inverse, n_L^2
  int nDense = 0;
  // Jacobi weight and coarse-correction scaling of the symmetric V(1,1)-cycle.  Piecewise-constant
  // prolongation under-estimates smooth error, and scaling the coarse correction (over-correction)
  // compensates; any positive scaling keeps the V-cycle SPD.  0.9 / 1.6 minimised the PCG
  // iterations on the jittered obstacle channel (105 -> 66 per outer step at 970k cells).
  double omega = 0.9;
  double corr = 1.6;
  cudaGraphExec_t graph = nullptr;  // captured V-cycle (see amg_capture_graph)
  int graphKernels = 0;
};
void amg_refresh(const LaunchCfg& lc, AmgDev& amg);  // Galerkin values + dense inverse
cudaError_t amg_capture_graph(const LaunchCfg& lc, const PcgArgs& a, AmgDev& amg);

}  // namespace anb
