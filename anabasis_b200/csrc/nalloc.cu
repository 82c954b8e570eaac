// Allocation-free patch-force integral (anb_patch_force_nalloc in include/anb.h).
//
// Some callers cannot allocate device memory at the point where they want the force: a host
// application that reserves the whole GPU for its own pool, code that runs while another
// component is recording a CUDA graph into the device's allocator, or a plugin whose memory
// budget is fixed when it is loaded.  This variant of the force reduction keeps its only scratch
// (per-block partial sums, the combined result and the arrival counter of the last-block
// combination) in one file-scope __device__ array, so a call performs no cudaMalloc, cudaFree or
// other allocating call.  Every GPU that loads the library holds the array until the process
// exits.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/anb.h"
#include "context_access.hpp"
#include "device.cuh"
#include "kernels.cuh"

namespace anb {
namespace {

constexpr int kNaBlocks = 1024;                 // partial sums for at most this many blocks
constexpr int kNaMaxFaces = kNaBlocks * kBlock;  // 262,144 patch faces: one face per thread
constexpr int kNaQ = 16;                        // quantities per partial (15 used)
constexpr int kNaResult = kNaBlocks * kNaQ;      // offset of the combined result (slot 15: written mark)
constexpr int kNaTicket = kNaResult + kNaQ;      // offset of the arrival counter (one double slot)
constexpr int kNaSize = kNaTicket + 2;           // 16,402 doubles = 131,216 bytes

// The scratch.  Host code only ever uses its device address from cudaGetSymbolAddress.  Before
// every launch the host clears the counter and the result slots on the call's stream.
static __device__ __align__(256) double g_forceScratch[kNaSize];

// Same per-face arithmetic as k_patch_force (main.cu:2869-2911 of the reference), one face per
// thread over at most kNaBlocks blocks (the partial-sum slots of the array); the last block to
// arrive combines the partials in block order and marks the result as written.
__global__ void __launch_bounds__(kBlock) k_patch_force_nalloc(DMesh m, int b0, int b1, int sign, double mu,
                                                               const double* bA, const double* bN, const double* U,
                                                               const double* P, double* scratch) {
  __shared__ double sm[kNaQ * 32];
  const int C = m.nCells;
  const unsigned maxMask = (1u << 11) | (1u << 12) | (1u << 13) | (1u << 14);
  double v[kNaQ];
  for (int q = 0; q < kNaQ; ++q) v[q] = ((maxMask >> q) & 1u) ? -1.0e308 : 0.0;
  const int b = b0 + blockIdx.x * blockDim.x + threadIdx.x;
  do {
    if (b >= b1) break;
    const int r = m.bOwner[b];
    const double A = bA[b];
    if (A <= 1.0e-300) break;
    double n0 = (double)sign * bN[3 * b], n1 = (double)sign * bN[3 * b + 1], n2 = (double)sign * bN[3 * b + 2];
    const double nm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    if (nm <= 1.0e-300) break;
    const double inv = 1.0 / nm;
    n0 *= inv;
    n1 *= inv;
    n2 *= inv;
    const double* d = m.bnd[b].d;
    const double dx0 = -d[0], dx1 = -d[1], dx2 = -d[2];
    double dn = dx0 * n0 + dx1 * n1 + dx2 * n2;
    if (dn <= 1.0e-14) dn = fabs(dn);
    if (dn <= 1.0e-14) dn = sqrt(dx0 * dx0 + dx1 * dx1 + dx2 * dx2);
    if (dn <= 1.0e-14) break;
    const double u0 = U[r], u1 = U[C + r], u2 = U[2 * C + r];
    const double Un = u0 * n0 + u1 * n1 + u2 * n2;
    const double t0 = u0 - Un * n0, t1 = u1 - Un * n1, t2 = u2 - Un * n2;
    const double Ut = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
    const double pr = P[r];
    const double nn[3] = {n0, n1, n2}, tt[3] = {t0, t1, t2};
    for (int q = 0; q < 3; ++q) {
      const double fp = -pr * nn[q] * A, fv = mu * tt[q] / dn * A;
      v[q] += fp;
      v[3 + q] += fv;
      v[6 + q] += fp + fv;
    }
    v[9] += A;
    v[10] += 1.0;
    v[11] = fmax(v[11], -dn);
    v[12] = fmax(v[12], dn);
    v[13] = fmax(v[13], Ut);
    v[14] = fmax(v[14], mu * Ut / dn);
  } while (false);
  Reducer red{scratch, reinterpret_cast<unsigned int*>(scratch + kNaTicket)};
  if (grid_reduce<kNaQ>(v, maxMask, red, sm) && threadIdx.x == 0) {
    double* out = scratch + kNaResult;
    for (int q = 0; q < 11; ++q) out[q] = v[q];
    const bool any = v[10] > 0.0;
    out[11] = any ? -v[11] : 0.0;
    out[12] = any ? v[12] : 0.0;
    out[13] = any ? v[13] : 0.0;
    out[14] = any ? v[14] : 0.0;
    out[15] = 1.0;
  }
}

// Device address of the scratch for each device, looked up once with that device current.
struct DeviceScratch {
  double* ptr = nullptr;
  bool ready = false;
};
std::mutex g_scratchMutex;
DeviceScratch g_scratch[64];

// Looks up the array's address on `device` (the current device).  The lookup is what places the
// library's module holding the array on the device (CUDA loads modules lazily), and the function
// attribute query loads the kernel's code, so both happen here and not at the first force call.
cudaError_t scratch_for_device(int device, double** out) {
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratchMutex);
  DeviceScratch& s = g_scratch[device];
  if (!s.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_forceScratch);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, k_patch_force_nalloc);
    if (e != cudaSuccess) return e;
    s.ptr = static_cast<double*>(p);
    s.ready = true;
  }
  *out = s.ptr;
  return cudaSuccess;
}

// Restores the caller's current device when the entry point returns.
struct DeviceRestore {
  int dev = -1;
  DeviceRestore() {
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  }
  ~DeviceRestore() {
    if (dev >= 0) cudaSetDevice(dev);
  }
};

}  // namespace

// Called by anb_create with the context's device current, while allocation is still allowed.
int nalloc_prepare_device(int device) {
  double* p = nullptr;
  return scratch_for_device(device, &p) == cudaSuccess ? 0 : 1;
}

}  // namespace anb

using namespace anb;

extern "C" int anb_patch_force_nalloc(anb_ctx* ctx, int patch, int normal_sign, anb_force_report* out) {
  if (!ctx || !out) return ANB_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  ForceView v;
  if (!context_force_view(ctx, patch, &v)) return ANB_OK;  // unknown patch: valid = 0, as anb_patch_force
  const int nFaces = v.b1 - v.b0;
  if (nFaces > kNaMaxFaces) {
    context_set_error(ctx, "anb_patch_force_nalloc: the patch has more than 262144 faces, the limit of the "
                           "allocation-free force integral (its static scratch holds 1024 block partials of "
                           "256 faces; use anb_patch_force)");
    return ANB_ERR_INVALID;
  }
  DeviceRestore restore;
  cudaError_t e = cudaSetDevice(v.device);
  double* scratch = nullptr;
  if (e == cudaSuccess) e = scratch_for_device(v.device, &scratch);
  // clear the arrival counter and the result slots on the call's stream (no allocation)
  if (e == cudaSuccess)
    e = cudaMemsetAsync(scratch + kNaResult, 0, sizeof(double) * (kNaSize - kNaResult), v.stream);
  if (e != cudaSuccess) {
    context_set_error(ctx, cudaGetErrorString(e));
    return ANB_ERR_CUDA;
  }
  const int blocks = std::max(1, (nFaces + kBlock - 1) / kBlock);
  g_launches += 1;
  k_patch_force_nalloc<<<blocks, kBlock, 0, v.stream>>>(v.dm, v.b0, v.b1, normal_sign, v.mu, v.bA, v.bN, v.U, v.P,
                                                        scratch);
  double h[kNaQ];
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, scratch + kNaResult, sizeof(h), cudaMemcpyDeviceToHost, v.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(v.stream);
  if (e != cudaSuccess) {
    context_set_error(ctx, cudaGetErrorString(e));
    return ANB_ERR_CUDA;
  }
  if (h[15] != 1.0) {  // the combining block never ran: a call overlapped this one on the device
    context_set_error(ctx, "anb_patch_force_nalloc: the result was not written (overlapping calls on one device?)");
    return ANB_ERR_CUDA;
  }
  out->valid = 1;
  for (int k = 0; k < 3; ++k) {
    out->Fp[k] = h[k];
    out->Fv[k] = h[3 + k];
    out->F[k] = h[6 + k];
  }
  out->area = h[9];
  out->n_faces = (int)h[10];
  out->min_wall_distance = h[11];
  out->max_wall_distance = h[12];
  out->max_ut = h[13];
  out->max_shear_mag = h[14];
  return ANB_OK;
}
