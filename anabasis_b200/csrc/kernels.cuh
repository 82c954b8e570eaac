// Launch wrappers for the SIMPLE kernels (implemented in kernels.cu).
#pragma once

#include "device.cuh"

#include <atomic>
#include <type_traits>
#include <vector>

namespace anb {

// Kernel families that can be timed with CUDA events (anb_profile_select in include/anb.h).
enum KernelFamily {
  kKfNone = 0, kKfGradient = 1, kKfMomentum = 2, kKfPressureRc = 3, kKfNonOrth = 4, kKfFluxFinal = 5,
  kKfBicgSpmv = 6, kKfPcgSpmv = 7, kKfAmgResid0 = 8, kKfAmgUp0 = 9, kKfAmgCoarse = 10, kKfPcgUpdate = 11,
  kKfBicgVector = 12, kKfMomentumSolve = 13, kKfPressureSolve = 14, kKfCount = 15
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
  int rowBlocks;   // most blocks a row-parallel (grid-stride) kernel gets; sizes the reduction partials
  cudaStream_t stream;
  Prof* prof = nullptr;
  const AlgoBytes* ab = nullptr;
  int nSM = 0;     // > 0: kernels launched through launch_rows get one full wave (see row_grid)
};

// Blocks of kBlock threads of `kernel` that fit on one SM at once (registers, shared memory);
// queried once per kernel.
int resident_blocks(const void* kernel);

// Grid of a grid-stride row kernel: one full wave of its resident blocks on every SM, at most
// `cap`.  With more blocks than fit, the blocks past the first wave run on a partly idle GPU at the
// end of the launch; the latency-bound SELL kernels lose up to 10 % to that tail.
inline int row_grid(const LaunchCfg& lc, const void* kernel, int cap) {
  if (lc.nSM <= 0) return cap;
  const int wave = resident_blocks(kernel) * lc.nSM;
  return wave > 0 && wave < cap ? wave : cap;
}

template <class... P, class... A>
inline void launch_rows(const LaunchCfg& lc, int cap, void (*kernel)(P...), A&&... args) {
  kernel<<<row_grid(lc, (const void*)kernel, cap), kBlock, 0, lc.stream>>>(static_cast<A&&>(args)...);
}

// Calls fn(std::integral_constant<int, W>) with the width class W (4, 6, 8 or 0 = generic) that a
// SELL matrix of rows of at most maxW slots is launched with.
template <class F>
inline void with_width(int maxW, F&& fn) {
  switch (launch_width_class(maxW)) {
    case 4: fn(std::integral_constant<int, 4>{}); break;
    case 6: fn(std::integral_constant<int, 6>{}); break;
    case 8: fn(std::integral_constant<int, 8>{}); break;
    default: fn(std::integral_constant<int, 0>{}); break;
  }
}

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

// M: storage type of the assembled matrix (double plain, float mixed precision); the right-hand
// sides, rAU and all arithmetic stay double.
template <class M>
struct MomArgsT {
  const double* U;    // 3*nCells old velocity (convecting velocity)
  const double* Q;    // 3*nCells field of the relaxation term (old field, or current iterate)
  const double* G;    // gradients of Q: [grad q0 | grad q1 | grad q2 | grad p], each 3*nCells SoA
  double rho, mu, uRelax;
  int relax;
  int rhsOnly;        // 1: right-hand sides only, relaxation from the stored relaxed diagonal
  M* val;
  M* diag;
  double* rhs;        // 3*nCells
  double* rau;
};
using MomArgs = MomArgsT<double>;
template <class M>
void launch_momentum(const LaunchCfg& lc, const DMesh& m, const MomArgsT<M>& a);

template <class M>
struct PresArgsT {
  const double* Us;   // 3*nCells momentum solution
  const double* P;
  const double* Gp;   // 3*nCells SoA
  const double* rau;
  double rho;
  M* val;
  M* diag;
  double* phiStar;    // nInternal + nBoundary
  double* divStar;
  double* b;          // first pressure right-hand side, -divStar
  double* pc;         // zeroed p'
  M* wdinv;           // optional: omega / diag for the AMG smoother
  double omega;
};
using PresArgs = PresArgsT<double>;
template <class M>
void launch_pressure_rc(const LaunchCfg& lc, const DMesh& m, const PresArgsT<M>& a);

// Scalar elliptic (libpoisson) and steady scalar transport (libscalar) systems on the SIMPLE
// layout.  Face arrays: internal faces in layout order and orientation, then boundary faces.
enum ScalarBc : uint8_t {
  kScalarDirichlet = 0,
  kScalarNeumann = 1,       // prescribed normal gradient (libpoisson Neumann, libscalar NeumannGradient)
  kScalarZeroGradient = 2,  // libscalar ZeroGradient
};
struct ScalarArgs {
  const double* phi;      // nCells
  const double* minv;     // 6 per cell, boundary-type dependent LSQ inverse
  const uint8_t* bcType;  // nBoundary (ScalarBc)
  const double* bcVal;    // nBoundary: Dirichlet value or normal gradient
  const double* bA;       // nBoundary face areas
  const double* bN;       // 3 per boundary face, unit outward normal
  const double* gammaF;   // nInternal + nBoundary
  const double* flux;     // nInternal + nBoundary face flux, or null (no convection)
  const double* src;      // nCells explicit source per unit volume (f or Su)
  const double* sp;       // nCells implicit source per unit volume, or null
  const double* grad;     // 3*nCells SoA gradient of phi
  int transport;          // 0: libpoisson elliptic rules, 1: libscalar transport rules
  int upwind;             // transport convection: 0 central, 1 upwind
  int nonorth;            // add the explicit non-orthogonal correction
  int refCell;            // layout cell fixed to refValue, -1 for none
  double refValue;
  double omega;           // weighted-Jacobi factor for the level-0 smoother weight
  double* g;              // gradient output (3*nCells)
  double* val;            // SELL off-diagonals
  double* diag;
  double* rhs;
  double* wdinv;          // omega / diag, or null
};
void launch_scalar_grad(const LaunchCfg& lc, const DMesh& m, const ScalarArgs& a);
void launch_scalar_assemble(const LaunchCfg& lc, const DMesh& m, const ScalarArgs& a);

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

// Extra pressure passes: b = -divCorr and dx = 0; y += s x.
void launch_pass_rhs(const LaunchCfg& lc, int n, const double* divCorr, double* b, double* dx);
void launch_add_scaled(const LaunchCfg& lc, int n, double s, const double* x, double* y);
// Cell fields between input and layout numbering: dst[q][i] = src[q][idx[i]], q < comps <= 4
struct PermuteArgs {
  const int* idx;
  const double* src[4];
  double* dst[4];
  int n, comps;
};
void launch_permute_cells(const LaunchCfg& lc, const PermuteArgs& a);
// out[2q], out[2q+1] = sum (after_q - before_q)^2, sum after_q^2 over n rows, q = 0..2 (device)
void launch_relchg3(const LaunchCfg& lc, int n, const double* before, const double* after, Reducer red,
                    double* out);

// Patch force (compute_patch_forces_wall_shear, main.cu:2828-2933) over boundary faces
// [b0, b1); out: Fp[3] Fv[3] F[3] area nFaces minDn maxDn maxUt maxShear (15 doubles).
void launch_patch_force(cudaStream_t s, const DMesh& m, int b0, int b1, int sign, double mu,
                        const double* bA, const double* bN, const double* U, const double* P, double* out);

// ---- Krylov ----------------------------------------------------------------------------
// T is the storage type of the matrix values and the solver vectors (double: plain method,
// float: mixed-precision inner solves); scalars, dot products and row sums are double.
template <class T>
struct BicgArgsT {
  DSellT<T> A;
  int nc;             // components (1..3), vectors are nc*n
  const T* b;
  T* x;
  T *r, *rh, *p, *v, *s, *t, *ph, *sh;
  double* sc;         // per component 8 scalars: rho, rhoN, alpha, omega, eps, rn, tsum, ssum
  int* fl;            // per component 4 ints: done, half, iters, converged; fl[12]: loop-graph trips
  double atol, rtol;
  int maxit;
  Reducer red;
  int precond;        // 0: Jacobi (ph = D^-1 p, sh = D^-1 s in the vector kernels); 1: the caller
                      // applies its preconditioner to p and s (bicg_iteration_precond)
};
using BicgArgs = BicgArgsT<double>;
template <class T>
void bicg_init(const LaunchCfg& lc, const BicgArgsT<T>& a);
template <class T>
void bicg_iteration(const LaunchCfg& lc, const BicgArgsT<T>& a);

// The BiCGSTAB iterations of a solve as one graph launch, for the arguments it was captured with.
template <class T>
struct BicgLoopT {
  cudaGraphExec_t exec = nullptr;
  BicgArgsT<T> args{};
  bool failed = false;  // capture failed once: the host loop runs
};
// After bicg_init: runs the (Jacobi-preconditioned) iterations as one launch of the loop graph,
// captured into `loop` on first use or when a's buffers changed, and returns true; returns false
// (nothing launched) with a preconditioner callback, when the graph cannot be built, or under
// ANB_NO_LOOP_GRAPH=1.  Iterations run in pairs; fl[12] counts the condition evaluations.
template <class T>
bool bicg_loop_launch(const LaunchCfg& lc, const BicgArgsT<T>& a, BicgLoopT<T>& loop);
template <class T>
void bicg_loop_release(BicgLoopT<T>& loop);

template <class T>
struct PcgArgsT {
  DSellT<T> A;
  const T* b;
  T* x;
  T *r, *z, *p0, *p1, *q;
  // AMG-preconditioned iterations keep the residual in two buffers (r, r2): the V-cycle's level-0
  // down sweep applies r_new = r - alpha q and x += alpha p itself, reading the old residual of
  // the neighbour rows from one buffer while it writes the new one into the other.
  T* r2;
  int mode;           // 0: PCG iteration; 1: plain preconditioner application z = M^-1 r (no update of
                      // x or r, no r.z reduction; fl[0] is the caller's done flag)
  double* sc;         // rz, alpha, beta, eps, rr, pq
  int* fl;            // done, iters, converged, first, loop-graph trips (pcg_capture_loop)
  double atol, rtol;
  int maxit;
  Reducer red;
};
using PcgArgs = PcgArgsT<double>;

// ---- AMG (aggregation, V-cycle) ------------------------------------------------------------
template <class T>
struct AmgLevelDevT {
  int n, nc;
  // matrix of this level: level 0 borrows the pressure matrix (SELL-32 slices in sliceOff); large
  // coarse levels are SELL-32 too (sliceOff, run by the level-0 kernels), small ones CSR (rowOff)
  const int* sliceOff;
  const int* rowOff;
  const int* col;
  T* val;
  T* diag;
  // restriction to the next level
  const int* agg;
  const int* memOff;
  const int* mem;
  // CSR levels: agg[col[k]] per stored entry, and the entry range {rowOff[i], rowOff[i + 1]} of
  // member mem[m] per member slot m; they take one dependent load out of the up and down sweeps
  const int* colAgg;
  const int2* memRow;
  const int* gOff;     // Galerkin gather for the next level's storage
  const int* gIdx;
  int nEntNext;        // next level's SELL storage entries
  // work vectors
  T *b, *x, *x2;
  T* wdinv;            // omega / diag (Jacobi smoother)
  int maxW;            // level 0: largest SELL slice width
};
template <class T>
struct AmgDevT {
  int nLevels = 0;
  AmgLevelDevT<T> lv[24];
  double* dense = nullptr;   // coarsest inverse, n_L^2, always double
  int nDense = 0;
  // Jacobi weight and coarse-correction scaling of the symmetric V(1,1)-cycle.  Piecewise-constant
  // prolongation under-estimates smooth error, and scaling the coarse correction (over-correction)
  // compensates; any positive scaling keeps the V-cycle SPD.  0.9 / 1.6 minimised the PCG
  // iterations on the jittered obstacle channel (105 -> 66 per outer step at 970k cells).
  double omega = 0.9;
  double corr = 1.6;
  // captured V-cycles (see amg_capture_graph): variant v reads the residual buffer v (r, r2) and
  // writes the other one, with the search direction p0 (v = 0) or p1 (v = 1)
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int graphKernels = 0;
  // the PCG iterations of a whole solve as one graph (see pcg_capture_loop), valid for the
  // arguments it was captured with
  cudaGraphExec_t loop = nullptr;
  PcgArgsT<T> loopArgs{};
  // Coarse tail: the CSR levels with at most tailRows rows and the dense level run as one
  // thread-block-cluster kernel of tailCluster CTAs (0: one launch per level and sweep).
  int tailRows = 0;
  int tailCluster = 0;
  // CSR levels of at most this many rows (above the tail) run their down sweep and restriction
  // as one kernel, warp per aggregate (same values; fewer launches, longer chains per warp)
  int fusedDownRows = 0;
};
using AmgLevelDev = AmgLevelDevT<double>;
using AmgDev = AmgDevT<double>;

template <class T>
void pcg_init(const LaunchCfg& lc, const PcgArgsT<T>& a);
// one iteration; `it` selects the p double buffer; amg == nullptr -> Jacobi
template <class T>
void pcg_iteration(const LaunchCfg& lc, const PcgArgsT<T>& a, int it, const AmgDevT<T>* amg);
// z = M^-1 r for the first iteration (and rz)
template <class T>
void pcg_precondition(const LaunchCfg& lc, const PcgArgsT<T>& a, const AmgDevT<T>* amg);
template <class T>
void amg_refresh(const LaunchCfg& lc, AmgDevT<T>& amg);  // Galerkin values + dense inverse
// z = M^-1 r with one V-cycle for arguments in mode 1 (r input, r2 scratch, z output, fl[0] a done
// flag that skips the application); captured into *graph on the first call when graph != nullptr
template <class T>
void amg_apply(const LaunchCfg& lc, const PcgArgsT<T>& a, const AmgDevT<T>* amg, cudaGraphExec_t* graph);
// One BiCGSTAB iteration with an external preconditioner: ph_c = M^-1 p_c after the p update and
// sh_c = M^-1 s_c after the s update, by apply(c, 0) and apply(c, 1) for the active components
template <class T>
void bicg_iteration_precond(const LaunchCfg& lc, const BicgArgsT<T>& a, void (*apply)(void* ctx, int c, int which),
                            void* ctx);
// Captures the two V-cycle variants for the PCG arguments a, then the solve loop
// (pcg_capture_loop); a loop that cannot be built is left out (the host loop runs instead).
template <class T>
cudaError_t amg_capture_graph(const LaunchCfg& lc, const PcgArgsT<T>& a, AmgDevT<T>& amg);
// After pcg_init and pcg_precondition: runs the solve's iterations as one launch of the loop graph
// and returns true, or returns false (nothing launched) when there is no loop graph for a.  The
// iterations run in pairs; fl[4] counts the graph's condition evaluations (2 (fl[4] - 1)
// iterations were enqueued on the device).
template <class T>
bool pcg_loop_launch(const LaunchCfg& lc, const PcgArgsT<T>& a, const AmgDevT<T>& amg);
// Destroys the captured V-cycles and the loop graph (the stream must be idle).
template <class T>
void amg_release_graphs(AmgDevT<T>& amg);
// Sets the coarse tail (levels of at most tailRows rows on one cluster; 0 = off) and picks its
// cluster size for this device.  Call before amg_capture_graph.
template <class T>
void amg_configure_tail(AmgDevT<T>& amg, int tailRows, cudaStream_t s);

// ---- mixed-precision defect correction (FP64 outer residual around FP32 inner solves) ------
// r = b - A x in double with the float matrix, r32 = r, per-component |r|^2 and |b|^2 in
// sc[8c+0..1]; done flags fl[4c] = |r| <= max(atol, rtol |b|) (nc components of n rows).
struct DefectArgs {
  DSellT<float> A;
  int nc;
  const double* b;
  const double* x;
  float* r32;
  double* sc;
  int* fl;
  const int* frozen;  // nc flags: components not solved (residual not needed), or null
  double atol, rtol;
  Reducer red;
};
void launch_defect(const LaunchCfg& lc, const DefectArgs& a);
// x += dx (nc*n), dx = 0
void launch_apply_correction(const LaunchCfg& lc, int n, int nc, double* x, float* dx);
// wdinv = omega / diag (n rows)
void launch_jacobi_weights(const LaunchCfg& lc, int n, double omega, const double* diag, double* wdinv);

// ---- steady residual, tangent and adjoint (kernels_adjoint.cu) -----------------------------
struct AdjArgs {
  const double* U;    // 3*nCells converged velocity
  const double* P;    // pressure
  const double* G;    // 12*nCells: gradients of u, v, w, p (BC values from DMesh::bVal)
  double* aP;         // unrelaxed momentum diagonal (written by adj_base)
  double* rau;        // rAU of the SIMPLE iteration (written by adj_base)
  double rho, mu, uRelax;
  int relax;
  Reducer red;
};
struct TanArgs {
  const double* dU;   // 3*nCells
  const double* dp;
  const double* dg;   // 3*nBoundary tangent of the Dirichlet velocity values (0 off the parameters)
  double dmu;
  const double* dG;   // 12*nCells gradients of du, dv, dw (BC values dg) and dp (BC values 0)
  double* daP;        // nCells work
};
struct AdjWork {
  const double* w;    // 4*nCells adjoint weights (u | v | w | continuity)
  double* abar;       // nCells work
  double* h;          // 12*nCells work
  double* gbar;       // 3*nBoundary adjoint of the Dirichlet velocity values, or null
  double* muBar;      // 1 (device)
};
struct ObjArgs {
  int b0, b1, sign;
  double dir[3];
  const double* bA;
  const double* bN;
  double* val;        // 2 (device): J, dJ/dmu at fixed (U, p)
};
void adj_base(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a);
void adj_residual(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a, double* R);
void adj_jvp(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a, const TanArgs& t, double* dR);
void adj_vjp(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a, const AdjWork& w, double* out);
void adj_objective(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a, const ObjArgs& o, double* out);
void adj_div_u(const LaunchCfg& lc, const DMesh& m, double rho, const double* v, double* y);
void adj_div_u_t(const LaunchCfg& lc, const DMesh& m, double rho, const double* w, double* Y);
// y = transpose of the LSQ gradient (field with Dirichlet bit dirBit) applied to fac*sc*s (s: 3C)
void adj_grad_t(const LaunchCfg& lc, const DMesh& m, const double* sc, double fac, const double* s, double* h,
                unsigned dirBit, double* y);
// x (3C) -= fac * sc * gp
void adj_sub_scaled_grad(const LaunchCfg& lc, int C, const double* sc, double fac, const double* gp, double* x);
void adj_permute(const LaunchCfg& lc, int n, const int* idx, const double* src, double* dst);
// out[j] = V_j . x for j < k (V: k vectors of length n, stride ld); partials: rowBlocks * k
void vec_mdot(const LaunchCfg& lc, size_t n, int k, const double* V, size_t ld, const double* x, double* partials,
              double* out);
// x = beta x + sum_j coef[j] V_j (coef on the device)
void vec_lincomb(const LaunchCfg& lc, size_t n, int k, const double* V, size_t ld, const double* coef, double beta,
                 double* x);

}  // namespace anb
