// Device-side data structures shared by the SIMPLE kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cstdlib>
#include <cuda_runtime.h>

namespace anb {

constexpr int kBlock = 256;
constexpr int kWarp = 32;

// One internal face, 64 bytes: two 32-byte sectors per gather.
struct __align__(16) FaceRec {
  double lam;     // clamped weight toward the neighbour (new orientation)
  double g;       // A / max(n.d, 1e-30)
  double t[3];    // S - g d  (non-orthogonal correction vector)
  double d[3];    // cc_N - cc_P
};

// One boundary face, 80 bytes.
struct __align__(16) BndRec {
  double g;       // A / max(n.d_b, 1e-30)
  double t[3];    // S - g d_b
  double S[3];    // area vector (outward)
  double d[3];    // x_f - cc_P
};

// Read-only mesh view passed by value to kernels.
struct DMesh {
  int nCells, nInternal, nBoundary, nSlices;
  int maxW;             // largest slice width (slots per row)
  const int* sliceOff;
  const int* col;
  const int* slotFace;
  const int* fOwner;    // internal faces in layout order: owner (lower new index) and neighbour
  const int* fNeigh;
  const FaceRec* face;
  const uint8_t* fFlags;
  // the face record of every slot, copied into slot order as 8 arrays of nEnt doubles (lam, g,
  // t[3], d[3]; zero on padding) with the face flags per slot: the slot loop of a warp then reads
  // its faces' geometry as contiguous runs instead of gathering 64-byte records by face index
  int nEnt;
  const double* slotGeom;
  const uint8_t* slotFlags;
  const int* bOwner;
  const BndRec* bnd;
  const uint8_t* bFlags;
  const int* cbOff;
  const int* cbList;
  const double* vol;
  const double* cc;     // 3 per cell
  const double* minv;   // 6 per cell
  // boundary conditions per boundary face: bit0 u, bit1 v, bit2 w, bit3 p Dirichlet
  const uint8_t* bType;
  const double* bVal;   // 4 * nBoundary: u | v | w | p face values
};

// First storage entry of row r in the SELL-32 pattern and the row's padded width.
__device__ __forceinline__ int row_base(const DMesh& m, int r, int& width) {
  const int s = r >> 5;
  const int b = __ldg(&m.sliceOff[s]);
  width = (__ldg(&m.sliceOff[s + 1]) - b) >> 5;
  return b + (r & 31);
}

__device__ __forceinline__ void load_face(const FaceRec* F, int f, double& lam, double& g, double t[3], double d[3]) {
  const double2* p = reinterpret_cast<const double2*>(F + f);
  const double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), e = __ldg(p + 3);
  lam = a.x; g = a.y; t[0] = b.x; t[1] = b.y; t[2] = c.x; d[0] = c.y; d[1] = e.x; d[2] = e.y;
}

// Face geometry of storage slot e (owner orientation, as in FaceRec).
__device__ __forceinline__ void load_slot(const DMesh& m, int e, double& lam, double& g, double t[3], double d[3]) {
  const double* s = m.slotGeom + e;
  const size_t n = (size_t)m.nEnt;
  lam = __ldg(s);
  g = __ldg(s + n);
  t[0] = __ldg(s + 2 * n);
  t[1] = __ldg(s + 3 * n);
  t[2] = __ldg(s + 4 * n);
  d[0] = __ldg(s + 5 * n);
  d[1] = __ldg(s + 6 * n);
  d[2] = __ldg(s + 7 * n);
}

__device__ __forceinline__ void load_bnd(const BndRec* B, int b, double& g, double t[3], double S[3], double d[3]) {
  const double2* p = reinterpret_cast<const double2*>(B + b);
  const double2 a = __ldg(p), c = __ldg(p + 1), e = __ldg(p + 2), h = __ldg(p + 3), k = __ldg(p + 4);
  g = a.x; t[0] = a.y; t[1] = c.x; t[2] = c.y; S[0] = e.x; S[1] = e.y; S[2] = h.x; d[0] = h.y; d[1] = k.x; d[2] = k.y;
}

// Generic SELL-32 sparse matrix (off-diagonals) + separate diagonal; values stored as T (double
// for the plain method, float for the mixed-precision inner solves), arithmetic in double.
template <class T>
struct DSellT {
  int n;
  const int* sliceOff;
  const int* col;
  const T* val;
  const T* diag;
  int maxW;        // largest slice width (slots per row); 0 = unknown
};
using DSell = DSellT<double>;

// Kernels specialised on a compile-time row width WM hold a row's slots in registers; this picks
// the smallest specialisation that covers the matrix (0: the generic loop).
__host__ __device__ inline int sell_width_class(int maxW) {
  return maxW <= 0 ? 0 : maxW <= 4 ? 4 : maxW <= 6 ? 6 : maxW <= 8 ? 8 : 0;
}

// Width class a launch wrapper instantiates.  ANB_SELL_WIDTH (4, 6 or 8) forces a wider class
// than the rows need, for measurements; a class narrower than maxW is ignored.  The arithmetic
// is the same in every class (padding slots are skipped).
inline int launch_width_class(int maxW) {
  static const int forced = [] {
    const char* s = std::getenv("ANB_SELL_WIDTH");
    return s ? std::atoi(s) : 0;
  }();
  const int wc = sell_width_class(maxW);
  if (wc > 0 && (forced == 4 || forced == 6 || forced == 8) && forced >= maxW) return forced;
  return wc;
}

// Cross-block deterministic reductions: each block writes a partial, the last block to arrive
// (atomic ticket) combines the partials in block order.
struct Reducer {
  double* partials;     // [maxBlocks * maxQ]
  unsigned int* ticket; // one counter, returns to 0 after each use
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Reduces NQ per-thread values over the block; result valid in thread 0.  ops: bit q set -> max.
template <int NQ>
__device__ __forceinline__ void block_reduce(double (&v)[NQ], unsigned maxMask, double* smem /*NQ*32*/) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = ((maxMask >> q) & 1u) ? warp_max(v[q]) : warp_sum(v[q]);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) smem[q * 32 + wid] = v[q];
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double x = lane < nw ? smem[q * 32 + lane] : (((maxMask >> q) & 1u) ? -1.0e308 : 0.0);
      v[q] = ((maxMask >> q) & 1u) ? warp_max(x) : warp_sum(x);
    }
  }
  __syncthreads();
}

// Block partial -> global; returns true in every thread of the last block, whose thread 0 then
// holds the grid-wide result in v.
template <int NQ>
__device__ __forceinline__ bool grid_reduce(double (&v)[NQ], unsigned maxMask, Reducer red, double* smem) {
  block_reduce<NQ>(v, maxMask, smem);
  __shared__ bool isLast;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) red.partials[(size_t)blockIdx.x * NQ + q] = v[q];
    __threadfence();
    unsigned t = atomicAdd(red.ticket, 1u);
    isLast = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!isLast) return false;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = ((maxMask >> q) & 1u) ? -1.0e308 : 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const double x = __ldcg(&red.partials[(size_t)b * NQ + q]);
      v[q] = ((maxMask >> q) & 1u) ? fmax(v[q], x) : v[q] + x;
    }
  }
  block_reduce<NQ>(v, maxMask, smem);
  if (threadIdx.x == 0) *red.ticket = 0u;
  return true;
}

}  // namespace anb
