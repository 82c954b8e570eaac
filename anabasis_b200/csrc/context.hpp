// Internal: the context behind the C ABI handle and the helpers shared by the files that
// implement entry points (anb_api.cu, adjoint_api.cu).  Not part of the public interface.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/anb.h"
#include "amg_setup.hpp"
#include "host_mesh.hpp"
#include "kernels.cuh"
#include "layout.hpp"

namespace anb {

struct AnbError : std::runtime_error {
  int code;
  AnbError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(call)                                                                                          \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess)                                                                                \
      throw AnbError(ANB_ERR_CUDA, std::string("CUDA error ") + cudaGetErrorString(e_) + " at " #call);   \
  } while (0)

// Device allocations owned by a context; freed together.
class DevArena {
 public:
  ~DevArena() { release(); }
  template <class T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    CK(cudaMalloc(&p, n * sizeof(T)));
    ptrs_.push_back(p);
    bytes_ += n * sizeof(T);
    return static_cast<T*>(p);
  }
  template <class T>
  T* upload(const std::vector<T>& h) {
    T* d = alloc<T>(h.size());
    if (!h.empty()) CK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
  }
  void release() {
    for (void* p : ptrs_) cudaFree(p);
    ptrs_.clear();
    bytes_ = 0;
  }
  size_t bytes() const { return bytes_; }

 private:
  std::vector<void*> ptrs_;
  size_t bytes_ = 0;
};

}  // namespace anb

using namespace anb;

namespace anb {
struct AdjointData;
}

struct anb_ctx {
  std::string err;
  anb_params prm{};
  HostMesh hm;
  Layout L;
  int C = 0, nI = 0, nB = 0, nEnt = 0;
  cudaStream_t stream = nullptr;
  LaunchCfg lc{};
  DevArena arena, amgArena;
  DMesh dm{};
  // face-slot lookup for diagnostics: storage entry of (owner row, neighbour col) and back
  std::vector<int> slotOwn, slotNei;
  // device buffers
  FaceRec* dFace = nullptr;
  BndRec* dBnd = nullptr;
  uint8_t* dBType = nullptr;
  double* dBVal = nullptr;
  double *dBA = nullptr, *dBN = nullptr;
  double *U = nullptr, *Us = nullptr, *P = nullptr, *Pc = nullptr, *rau = nullptr;
  double *G = nullptr, *Gc = nullptr;
  double *mval = nullptr, *mdiag = nullptr, *rhs = nullptr;
  double *pval = nullptr, *pdiag = nullptr, *pb = nullptr, *divStar = nullptr, *divCorr = nullptr;
  double *phiStar = nullptr, *phi = nullptr;
  double* UsPrev = nullptr;   // momentum iterates before a re-solve (3*C; only with nVelNonOrthCorr > 0)
  double *bw[8] = {nullptr};  // BiCGSTAB work vectors (3*C each)
  double *pr = nullptr, *pz = nullptr, *pp0 = nullptr, *pp1 = nullptr, *pq = nullptr, *pdx = nullptr;
  // second PCG residual buffer and the PCG iterate at a fixed address (the captured V-cycles update
  // both in place); solve_pressure copies the caller's x in and out
  double *pr2 = nullptr, *pxw = nullptr;
  double* pwdinv = nullptr;   // omega / pressure diagonal (level-0 smoother)
  double* scal = nullptr;     // device scalars
  int* flags = nullptr;
  double* stats = nullptr;
  double* forceOut = nullptr;
  Reducer red{};
  // pinned host mirrors
  int* hFlags = nullptr;
  // flags of the solves that ran as loop graphs in the current step, copied here asynchronously
  // and read after the step's one synchronisation (kDeferSlots slots of kDeferInts ints)
  int* hDefer = nullptr;
  int nDefer = 0;
  double* hScal = nullptr;
  // cell fields cross the host/device boundary through 4 * nCells pinned doubles (hStage) and
  // 4 * nCells device doubles in input numbering (dStage), permuted on the device by the new->old
  // (dN2O) and old->new (dO2N) cell maps; stageEv marks the chunks of a download
  static constexpr int kStageEvents = 64;
  double* hStage = nullptr;
  double* dStage = nullptr;
  int *dN2O = nullptr, *dO2N = nullptr;
  cudaEvent_t stageEv[kStageEvents] = {};
  // state
  bool bcSet = false, stateSet = false, pZeroBC = true;
  long long outerStep = 0;
  int lastMomIts = 8, lastPIts = 8;
  // AMG
  bool amgBuilt = false;
  AmgDev amg;
  std::vector<AmgLevelHost> amgHost;
  // measurement
  Prof prof;
  AlgoBytes ab;
  // mixed precision (precision == ANB_PRECISION_MIXED): float matrices and inner-solver vectors
  bool mixed = false;
  float *mval32 = nullptr, *mdiag32 = nullptr, *pval32 = nullptr, *pdiag32 = nullptr, *pwdinv32 = nullptr;
  float* bw32[8] = {nullptr};
  float *r32 = nullptr, *dx32 = nullptr;                     // 3*nCells each
  float *pr32 = nullptr, *pz32 = nullptr, *pp0_32 = nullptr, *pp1_32 = nullptr, *pq32 = nullptr, *pr2_32 = nullptr;
  AmgDevT<float> amg32;
  double innerRtol = 1e-4;    // relative reduction asked of one FP32 inner solve at most
  // scalar-library solves (allocated on first use)
  DevArena scalarArena;
  double *sMinv = nullptr, *sBcVal = nullptr, *sGamma = nullptr, *sFlux = nullptr, *sSrc = nullptr,
         *sSp = nullptr, *sPhi = nullptr, *sGrad = nullptr;
  uint8_t* sBcType = nullptr;
  // steady sensitivities (adjoint_api.cu, allocated on first use)
  anb::AdjointData* adj = nullptr;
  // anb_create wall seconds: copy-in + topology, geometry, layout, device build + upload
  double setupSec[4] = {0, 0, 0, 0};
  // momentum AMG preconditioner (mom_amg = 1): hierarchy of the momentum matrix, level-0 Jacobi
  // weights, V-cycle arguments and graphs per (component, p or s) application, scratch vector
  bool momAmgBuilt = false;
  AmgDev amgMom;
  std::vector<AmgLevelHost> amgMomHost;
  DevArena amgMomArena;
  double *mwdinv = nullptr, *momScratch = nullptr, *momSc = nullptr;
  PcgArgs momArgs[6] = {};
  cudaGraphExec_t momGraph[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  // momentum BiCGSTAB iterations as one graph launch (FP64, and the FP32 inner solves)
  BicgLoopT<double> momLoop;
  BicgLoopT<float> momLoop32;
};

namespace anb {

constexpr int kScalBicg = 0;    // 3 * 8
constexpr int kScalPcg = 24;    // 8
constexpr int kFlagBicg = 0;    // 3 * 4
constexpr int kFlagPcg = 32;    // 8: done, iterations, converged, first, loop-graph trips
constexpr int kFlagCount = 40;  // ints in anb_ctx::flags (and hFlags)
constexpr int kDeferSlots = 64;
constexpr int kDeferInts = 16;
constexpr int kScalRelchg = 56; // 6: momentum relative-change sums

int fail(anb_ctx* c, const AnbError& e);

// Every entry point leaves the caller's current device as it found it (the calls select the
// context's device themselves).
struct CallerDevice {
  int dev = -1;
  CallerDevice() {
    if (cudaGetDevice(&dev) != cudaSuccess) {
      cudaGetLastError();
      dev = -1;
    }
  }
  ~CallerDevice() {
    if (dev >= 0) cudaSetDevice(dev);
  }
};

template <class F>
int guarded(anb_ctx* c, F&& f) {
  CallerDevice keep;
  try {
    return f();
  } catch (const AnbError& e) {
    return fail(c, e);
  } catch (const std::bad_alloc&) {
    if (c) c->err = "host allocation failed";
    return ANB_ERR_INVALID;
  } catch (const std::exception& e) {
    if (c) c->err = e.what();
    return ANB_ERR_MESH;
  }
}

// comps <= 4 cell fields in input numbering <-> device arrays in layout numbering; the
// single-pointer forms take comps consecutive nCells blocks on the device
void upload_cells(anb_ctx* c, const double* const* src, double* const* dst, int comps);
void upload_cells(anb_ctx* c, const double* const* src, double* dst, int comps);
void download_cells(anb_ctx* c, const double* const* src, double* const* dst, int comps);
void download_cells(anb_ctx* c, const double* src, double* const* dst, int comps);
DSell mom_sell(const anb_ctx* c);
DSell p_sell(const anb_ctx* c);
void grad(anb_ctx* c, int nf, const double* const* phi, const unsigned char* bits, double* const* out);
void poll(anb_ctx* c, const int* dflags, int count);
PcgArgs pcg_args(anb_ctx* c, const double* b, double rtol);
void solve_pressure(anb_ctx* c, const double* b, double* x, double rtol, int* its, bool* conv);
void ensure_amg(anb_ctx* c);
void launch_mom(anb_ctx* c, const double* Q, int rhsOnly);
void release_amg(anb_ctx* c);
void check_ready(anb_ctx* c);
void adjoint_release(anb_ctx* c);

}  // namespace anb
