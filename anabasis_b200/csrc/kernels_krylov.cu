// Krylov solvers and the aggregation-AMG V-cycle (sm_100a), standing in for the reference's
// HYPRE BiCGSTAB+DiagScale momentum solve (main.cu:2553-2576) and PCG+BoomerAMG pressure solve
// (main.cu:2224-2273, 2617-2676).
//
// All scalars stay on the device: every reduction ends in the last block of its kernel
// (deterministic block-order combination), which also advances the recurrence scalars and the
// convergence flags.  Kernels return immediately once their system is converged, so the host
// can enqueue several iterations between polls without changing the arithmetic.
//
// Every kernel is a template over T, the storage type of matrix values and solver vectors:
// double for the plain method, float for the inner solves of the mixed-precision method (inside
// an FP64 defect correction, bottom of this file).  Row sums, dot products and recurrence
// scalars are double in both.
#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace anb {
namespace {

namespace cg = cooperative_groups;

template <class T>
__device__ __forceinline__ double ld(const T* p) {
  return (double)__ldg(p);
}

// y = (D + Off) x for one row of a SELL-32 matrix
template <class T, class X>
__device__ __forceinline__ double sell_row(const DSellT<T>& A, int r, const X* x) {
  const int s = r >> 5;
  const int b = __ldg(&A.sliceOff[s]) + (r & 31);
  const int W = (__ldg(&A.sliceOff[s + 1]) - __ldg(&A.sliceOff[s])) >> 5;
  double y = (double)A.diag[r] * (double)x[r];
#pragma unroll 4
  for (int k = 0; k < W; ++k) {
    const int e = b + (k << 5);
    y += ld(&A.val[e]) * (double)x[__ldg(&A.col[e])];
  }
  return y;
}

// y_c = (D + Off) x_c for up to three vectors sharing one pass over the matrix row
template <class T>
__device__ __forceinline__ void sell_row3(const DSellT<T>& A, int r, const T* x, size_t n, const bool* act, int nc,
                                          double* y) {
  const int s = r >> 5;
  const int b = __ldg(&A.sliceOff[s]) + (r & 31);
  const int W = (__ldg(&A.sliceOff[s + 1]) - __ldg(&A.sliceOff[s])) >> 5;
  const double d = (double)A.diag[r];
#pragma unroll
  for (int c = 0; c < 3; ++c) y[c] = (c < nc && act[c]) ? d * (double)x[c * n + r] : 0.0;
#pragma unroll 2
  for (int k = 0; k < W; ++k) {
    const int e = b + (k << 5);
    const double v = ld(&A.val[e]);
    const int j = __ldg(&A.col[e]);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if (c < nc && act[c]) y[c] += v * (double)x[c * n + j];
  }
}

// Row r's slots in registers, for a compile-time bound WM on the slice width: every column and
// value load of the row is issued before the first gather, so a row costs two dependent memory
// round trips instead of two per unrolled group.  Slots past the row's slice width are
// (column r, value 0) and read nothing.
template <int WM, class T>
__device__ __forceinline__ void sell_regs(const int* sliceOff, const int* col, const T* val, int r, int (&c)[WM],
                                          double (&v)[WM]) {
  const int s = r >> 5;
  const int b0 = __ldg(&sliceOff[s]);
  const int W = (__ldg(&sliceOff[s + 1]) - b0) >> 5;
  const int b = b0 + (r & 31);
#pragma unroll
  for (int k = 0; k < WM; ++k) {
    c[k] = r;
    v[k] = 0.0;
    if (k < W) {
      c[k] = __ldg(&col[b + (k << 5)]);
      v[k] = ld(&val[b + (k << 5)]);
    }
  }
}

// sell_row3 with the row in registers
template <int WM, class T>
__device__ __forceinline__ void sell_row3_regs(const DSellT<T>& A, int r, const T* x, size_t n, const bool* act, int nc,
                                               double* y) {
  int c[WM];
  double v[WM];
  sell_regs<WM>(A.sliceOff, A.col, A.val, r, c, v);
  const double d = (double)A.diag[r];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (!(q < nc && act[q])) {
      y[q] = 0.0;
      continue;
    }
    const T* xq = x + q * n;
    double acc = d * (double)xq[r];
#pragma unroll
    for (int k = 0; k < WM; ++k) acc += v[k] * (double)xq[c[k]];
    y[q] = acc;
  }
}

template <int WM, class T>
__device__ __forceinline__ void row3(const DSellT<T>& A, int r, const T* x, size_t n, const bool* act, int nc,
                                     double* y) {
  if constexpr (WM == 0) sell_row3(A, r, x, n, act, nc, y);
  else sell_row3_regs<WM>(A, r, x, n, act, nc, y);
}

// ---------------------------------------------------------------- BiCGSTAB, nc components
// scalars per component c: sc[8c + 0..7] = rho, rhoN, alpha, omega, eps, rn, -, -
// flags per component c:   fl[4c + 0..3] = done, half, iters, converged
// Component loops run over the constant bound 3 with `c < nc` as a guard: with a run-time bound
// the per-component arrays (flags, scalars, partial sums) are indexed dynamically and live in
// local memory, which cost ~0.5 ms per SIMPLE step at 970k cells.

__device__ __forceinline__ bool all_done(const int* fl, int nc) {
  for (int c = 0; c < nc; ++c)
    if (!fl[4 * c]) return false;
  return true;
}

// Condition of the BiCGSTAB loop graph (one thread): go on while a component is not done, for at
// most maxTrips evaluations (fl[12], zeroed by k_bicg_init, counts them).
__global__ void k_bicg_loop_cond(cudaGraphConditionalHandle h, int* fl, int nc, int maxTrips) {
  const int t = fl[12] + 1;
  fl[12] = t;
  cudaGraphSetConditional(h, (!all_done(fl, nc) && t < maxTrips) ? 1u : 0u);
}

template <class T, int WM>
__global__ void __launch_bounds__(kBlock) k_bicg_init(BicgArgsT<T> a) {
  __shared__ double sm[6 * 32];
  const int n = a.A.n;
  const bool all[3] = {true, true, true};
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double ax[3];  // (A x)_r of every component, one pass over the row (same terms, same order)
    row3<WM>(a.A, r, a.x, (size_t)n, all, a.nc, ax);
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      const size_t o = (size_t)c * n;
      const double bb = (double)a.b[o + r];
      const double rr = bb - ax[c];
      a.r[o + r] = (T)rr;
      a.rh[o + r] = (T)rr;
      a.p[o + r] = T(0);
      a.v[o + r] = T(0);
      acc[2 * c] += rr * rr;
      acc[2 * c + 1] += bb * bb;
    }
  }
  if (grid_reduce<6>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      double* s = a.sc + 8 * c;
      int* f = a.fl + 4 * c;
      const double bn = sqrt(acc[2 * c + 1]);
      s[4] = fmax(a.atol, a.rtol * bn);
      s[5] = sqrt(acc[2 * c]);
      s[0] = 1.0;
      s[1] = acc[2 * c];
      s[2] = 1.0;
      s[3] = 1.0;
      f[0] = (s[5] <= s[4]) ? 1 : 0;
      f[1] = 0;
      f[2] = 0;
      f[3] = f[0];
    }
    a.fl[12] = 0;
  }
}

// p = r + beta (p - omega v); ph = D^-1 p
template <class T>
__global__ void __launch_bounds__(kBlock) k_bicg_p(BicgArgsT<T> a) {
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  double beta[3], om[3];
  bool act[3];
  _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
    const double* s = a.sc + 8 * c;
    act[c] = !a.fl[4 * c];
    beta[c] = (s[1] / s[0]) * (s[2] / s[3]);
    om[c] = s[3];
  }
  // every load of a row (all components) is issued before its stores, which the compiler must
  // otherwise assume alias the next component's inputs
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double dinv = 1.0 / (double)a.A.diag[r];
    double rv[3], pv[3], vv[3];
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      const size_t i = (size_t)c * n + r;
      rv[c] = ld(&a.r[i]);
      pv[c] = (double)a.p[i];
      vv[c] = ld(&a.v[i]);
    }
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      const size_t i = (size_t)c * n + r;
      const double pn = rv[c] + beta[c] * (pv[c] - om[c] * vv[c]);
      a.p[i] = (T)pn;
      if (!a.precond) a.ph[i] = (T)(dinv * pn);
    }
  }
}

// v = A ph ; alpha = rhoN / (rh . v) ; rho = rhoN
template <class T, int WM>
__global__ void __launch_bounds__(kBlock) k_bicg_v(BicgArgsT<T> a) {
  __shared__ double sm[3 * 32];
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  bool act[3];
  _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) act[c] = !a.fl[4 * c];
  double acc[3] = {0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double y[3];
    row3<WM>(a.A, r, a.ph, (size_t)n, act, a.nc, y);
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      const size_t o = (size_t)c * n;
      a.v[o + r] = (T)y[c];
      acc[c] += (double)a.rh[o + r] * y[c];
    }
  }
  if (grid_reduce<3>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      double* s = a.sc + 8 * c;
      s[2] = acc[c] != 0.0 ? s[1] / acc[c] : 0.0;
      s[0] = s[1];
      if (acc[c] == 0.0) {  // breakdown: stop this component
        a.fl[4 * c] = 1;
        a.fl[4 * c + 3] = 0;
      }
    }
  }
}

// s = r - alpha v ; sh = D^-1 s ; early exit if |s| <= eps
template <class T>
__global__ void __launch_bounds__(kBlock) k_bicg_s(BicgArgsT<T> a) {
  __shared__ double sm[3 * 32];
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  bool act[3];
  double al[3];
  _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
    act[c] = !a.fl[4 * c];
    al[c] = a.sc[8 * c + 2];
  }
  double acc[3] = {0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double dinv = 1.0 / (double)a.A.diag[r];
    double rv[3], vv[3];
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {  // loads first, as in k_bicg_p
      if (!act[c]) continue;
      const size_t i = (size_t)c * n + r;
      rv[c] = ld(&a.r[i]);
      vv[c] = ld(&a.v[i]);
    }
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      const size_t i = (size_t)c * n + r;
      const double sv = rv[c] - al[c] * vv[c];
      a.s[i] = (T)sv;
      if (!a.precond) a.sh[i] = (T)(dinv * sv);
      acc[c] += sv * sv;
    }
  }
  if (grid_reduce<3>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      if (sqrt(acc[c]) <= a.sc[8 * c + 4]) a.fl[4 * c + 1] = 1;
    }
  }
}

// t = A sh ; omega = (t.s)/(t.t)
template <class T, int WM>
__global__ void __launch_bounds__(kBlock) k_bicg_t(BicgArgsT<T> a) {
  __shared__ double sm[6 * 32];
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  bool act[3];
  _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) act[c] = !a.fl[4 * c] && !a.fl[4 * c + 1];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double y[3];
    row3<WM>(a.A, r, a.sh, (size_t)n, act, a.nc, y);
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      const size_t o = (size_t)c * n;
      const double tv = y[c];
      a.t[o + r] = (T)tv;
      acc[2 * c] += tv * (double)a.s[o + r];
      acc[2 * c + 1] += tv * tv;
    }
  }
  if (grid_reduce<6>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      a.sc[8 * c + 3] = acc[2 * c + 1] > 0.0 ? acc[2 * c] / acc[2 * c + 1] : 0.0;
    }
  }
}

// x += alpha ph + omega sh ; r = s - omega t ; convergence
template <class T>
__global__ void __launch_bounds__(kBlock) k_bicg_x(BicgArgsT<T> a) {
  __shared__ double sm[6 * 32];
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  bool act[3], half[3];
  double al[3], om[3];
  _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
    act[c] = !a.fl[4 * c];
    half[c] = a.fl[4 * c + 1] != 0;
    al[c] = a.sc[8 * c + 2];
    om[c] = a.sc[8 * c + 3];
  }
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double xv[3], phv[3], shv[3], sv[3], tv[3], rhv[3];
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {  // loads first, as in k_bicg_p
      if (!act[c]) continue;
      const size_t i = (size_t)c * n + r;
      xv[c] = (double)a.x[i];
      phv[c] = ld(&a.ph[i]);
      if (!half[c]) {
        shv[c] = ld(&a.sh[i]);
        sv[c] = ld(&a.s[i]);
        tv[c] = ld(&a.t[i]);
        rhv[c] = ld(&a.rh[i]);
      }
    }
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      const size_t i = (size_t)c * n + r;
      if (half[c]) {
        a.x[i] = (T)(xv[c] + al[c] * phv[c]);
      } else {
        a.x[i] = (T)(xv[c] + al[c] * phv[c] + om[c] * shv[c]);
        const double rr = sv[c] - om[c] * tv[c];
        a.r[i] = (T)rr;
        acc[2 * c] += rr * rr;
        acc[2 * c + 1] += rhv[c] * rr;
      }
    }
  }
  if (grid_reduce<6>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      double* s = a.sc + 8 * c;
      int* f = a.fl + 4 * c;
      f[2] += 1;
      if (half[c]) {
        f[0] = 1;
        f[3] = 1;
        continue;
      }
      s[5] = sqrt(acc[2 * c]);
      s[1] = acc[2 * c + 1];
      if (s[5] <= s[4]) {
        f[0] = 1;
        f[3] = 1;
      } else if (f[2] >= a.maxit || s[3] == 0.0) {
        f[0] = 1;
        f[3] = 0;
      }
    }
  }
}

// ---------------------------------------------------------------- PCG
// sc: 0 rz, 1 alpha, 2 beta, 3 eps, 4 rr, 5 pq ; fl: 0 done, 1 iters, 2 converged, 3 first

template <class T, int WM>
__global__ void __launch_bounds__(kBlock) k_pcg_init(PcgArgsT<T> a) {
  __shared__ double sm[2 * 32];
  const int n = a.A.n;
  const bool all[1] = {true};
  double acc[2] = {0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double bb = (double)a.b[r];
    double ax[3];
    row3<WM>(a.A, r, a.x, (size_t)n, all, 1, ax);  // the row in registers for WM > 0, same sum
    const double rr = bb - ax[0];
    a.r[r] = (T)rr;
    acc[0] += rr * rr;
    acc[1] += bb * bb;
  }
  if (grid_reduce<2>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    a.sc[3] = fmax(a.atol, a.rtol * sqrt(acc[1]));
    a.sc[4] = acc[0];
    a.sc[2] = 0.0;
    a.fl[0] = sqrt(acc[0]) <= a.sc[3] ? 1 : 0;
    a.fl[1] = 0;
    a.fl[2] = a.fl[0];
    a.fl[3] = 1;
    a.fl[4] = 0;
  }
}

// Jacobi preconditioner z = D^-1 r with rz (used when the AMG is off)
template <class T>
__global__ void __launch_bounds__(kBlock) k_pcg_jacobi(PcgArgsT<T> a) {
  __shared__ double sm[32];
  if (a.fl[0]) return;
  const int n = a.A.n;
  double acc[1] = {0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double z = (double)a.r[r] / (double)a.A.diag[r];
    a.z[r] = (T)z;
    acc[0] += (double)a.r[r] * z;
  }
  if (grid_reduce<1>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    const double rzOld = a.sc[0];
    a.sc[2] = a.fl[3] ? 0.0 : acc[0] / rzOld;
    a.sc[0] = acc[0];
  }
}

// pNew = z + beta pOld (rows and, on the fly, their neighbours); q = A pNew; alpha = rz / (p.q)
template <class T, int WM>
__global__ void __launch_bounds__(kBlock) k_pcg_pq(PcgArgsT<T> a, const T* pOld, T* pNew) {
  __shared__ double sm[32];
  if (a.fl[0]) return;
  const int n = a.A.n;
  // first iteration: p = z, and p_old is not read (it may hold anything, NaN included)
  const bool first = a.fl[3] != 0;
  const double beta = first ? 0.0 : a.sc[2];
  double acc[1] = {0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double pr = first ? (double)a.z[r] : (double)(T)((double)a.z[r] + beta * (double)pOld[r]);
    double q = (double)a.A.diag[r] * pr;
    if constexpr (WM == 0) {
      const int s = r >> 5;
      const int b = __ldg(&a.A.sliceOff[s]) + (r & 31);
      const int W = (__ldg(&a.A.sliceOff[s + 1]) - __ldg(&a.A.sliceOff[s])) >> 5;
      for (int k = 0; k < W; ++k) {
        const int e = b + (k << 5);
        const int c = __ldg(&a.A.col[e]);
        q += (double)a.A.val[e] * (first ? (double)a.z[c] : (double)(T)((double)a.z[c] + beta * (double)pOld[c]));
      }
    } else {
      int c[WM];
      double v[WM];
      sell_regs<WM>(a.A.sliceOff, a.A.col, a.A.val, r, c, v);
#pragma unroll
      for (int k = 0; k < WM; ++k)
        q += v[k] * (first ? (double)a.z[c[k]] : (double)(T)((double)a.z[c[k]] + beta * (double)pOld[c[k]]));
    }
    pNew[r] = (T)pr;
    a.q[r] = (T)q;
    acc[0] += pr * q;
  }
  if (grid_reduce<1>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    a.sc[5] = acc[0];
    a.sc[1] = acc[0] != 0.0 ? a.sc[0] / acc[0] : 0.0;
    a.fl[3] = 0;
  }
}

// Iteration count and convergence test on |r|^2 = rr (last block, thread 0).
template <class T>
__device__ __forceinline__ void pcg_converged(const PcgArgsT<T>& a, double rr) {
  a.sc[4] = rr;
  a.fl[1] += 1;
  if (sqrt(rr) <= a.sc[3]) {
    a.fl[0] = 1;
    a.fl[2] = 1;
  } else if (a.fl[1] >= a.maxit || a.sc[5] == 0.0) {
    a.fl[0] = 1;
    a.fl[2] = 0;
  }
}

// x += alpha p ; r -= alpha q ; convergence test on |r|
template <class T>
__global__ void __launch_bounds__(kBlock) k_pcg_xr(PcgArgsT<T> a, const T* p) {
  __shared__ double sm[32];
  if (a.fl[0]) return;
  const int n = a.A.n;
  const double al = a.sc[1];
  double acc[1] = {0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    a.x[r] = (T)__fma_rn(al, (double)p[r], (double)a.x[r]);
    const double rr = __fma_rn(-al, (double)a.q[r], (double)a.r[r]);
    a.r[r] = (T)rr;
    acc[0] += rr * rr;
  }
  if (grid_reduce<1>(acc, 0u, a.red, sm) && threadIdx.x == 0) pcg_converged(a, acc[0]);
}

// Condition of the PCG loop graph (one thread): go on while the solve is not done, for at most
// maxTrips evaluations (fl[4], zeroed by k_pcg_init, counts them).
__global__ void k_pcg_loop_cond(cudaGraphConditionalHandle h, int* fl, int maxTrips) {
  const int t = fl[4] + 1;
  fl[4] = t;
  cudaGraphSetConditional(h, (fl[0] == 0 && t < maxTrips) ? 1u : 0u);
}

// ---------------------------------------------------------------- AMG V-cycle
// Down, part 1: weighted-Jacobi pre-smoothing from zero (x = w D^-1 b) fused with the residual
// r = b - A x (neighbour x computed on the fly); thread per row, SELL-coalesced.  r goes to x2,
// which is free until the up sweep.
template <class T, int WM>
__global__ void __launch_bounds__(kBlock) k_amg_resid(const int* done, AmgLevelDevT<T> f, double omega) {
  if (*done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < f.n; i += gridDim.x * blockDim.x) {
    const double di = ld(&f.diag[i]);
    const double bi = ld(&f.b[i]);
    const double xi = ld(&f.wdinv[i]) * bi;
    double ax = di * xi;
    if constexpr (WM == 0) {
      const int s = i >> 5;
      const int b = __ldg(&f.sliceOff[s]) + (i & 31);
      const int W = (__ldg(&f.sliceOff[s + 1]) - __ldg(&f.sliceOff[s])) >> 5;
#pragma unroll 4
      for (int k = 0; k < W; ++k) {
        const int e = b + (k << 5);
        const int j = __ldg(&f.col[e]);
        ax += ld(&f.val[e]) * (ld(&f.wdinv[j]) * ld(&f.b[j]));
      }
    } else {
      int c[WM];
      double v[WM];
      sell_regs<WM>(f.sliceOff, f.col, f.val, i, c, v);
#pragma unroll
      for (int k = 0; k < WM; ++k) ax += v[k] * (ld(&f.wdinv[c[k]]) * ld(&f.b[c[k]]));
    }
    f.x[i] = (T)xi;
    f.x2[i] = (T)(bi - ax);
  }
}

// Level-0 down sweep fused with the update of the PCG iteration before it: r_new = r - alpha q and
// x += alpha p on the row's own entries, |r_new|^2 with the convergence test in the last block,
// then the pre-smoothing x0 = w D^-1 r_new and the residual x2 = r_new - A x0.  The neighbours'
// r_new come from their old residual and q, rounded to T as their own rows store them, so the
// values are those of a separate update kernel followed by k_amg_resid.  The old residual is read
// from rIn and the new one written to rOut (other rows still read rIn).  Right after pcg_init
// (flag "first") there is no update: r_new = r.
template <class T, int WM>
__global__ void __launch_bounds__(kBlock) k_amg_resid0(PcgArgsT<T> a, AmgLevelDevT<T> f, const T* rIn, T* rOut,
                                                       const T* p) {
  __shared__ double sm[32];
  if (a.fl[0]) return;
  const bool upd = a.mode == 0 && a.fl[3] == 0;
  const double al = upd ? a.sc[1] : 0.0;
  double acc[1] = {0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < f.n; i += gridDim.x * blockDim.x) {
    double ri;
    if (upd) {
      const double rr = __fma_rn(-al, ld(&a.q[i]), ld(&rIn[i]));
      acc[0] += rr * rr;
      ri = (double)(T)rr;
      a.x[i] = (T)__fma_rn(al, (double)p[i], (double)a.x[i]);
    } else {
      ri = ld(&rIn[i]);
    }
    rOut[i] = (T)ri;
    const double di = ld(&f.diag[i]);
    const double xi = ld(&f.wdinv[i]) * ri;
    double ax = di * xi;
    if constexpr (WM == 0) {
      const int s = i >> 5;
      const int b = __ldg(&f.sliceOff[s]) + (i & 31);
      const int W = (__ldg(&f.sliceOff[s + 1]) - __ldg(&f.sliceOff[s])) >> 5;
#pragma unroll 4
      for (int k = 0; k < W; ++k) {
        const int e = b + (k << 5);
        const int j = __ldg(&f.col[e]);
        const double rj = upd ? (double)(T)__fma_rn(-al, ld(&a.q[j]), ld(&rIn[j])) : ld(&rIn[j]);
        ax += ld(&f.val[e]) * (ld(&f.wdinv[j]) * rj);
      }
    } else {
      int c[WM];
      double v[WM];
      sell_regs<WM>(f.sliceOff, f.col, f.val, i, c, v);
#pragma unroll
      for (int k = 0; k < WM; ++k) {
        const double rj = upd ? (double)(T)__fma_rn(-al, ld(&a.q[c[k]]), ld(&rIn[c[k]])) : ld(&rIn[c[k]]);
        ax += v[k] * (ld(&f.wdinv[c[k]]) * rj);
      }
    }
    f.x[i] = (T)xi;
    f.x2[i] = (T)(ri - ax);
  }
  if (!upd) return;  // uniform over the grid
  if (grid_reduce<1>(acc, 0u, a.red, sm) && threadIdx.x == 0) pcg_converged(a, acc[0]);
}

constexpr int kCoarseLanes = 8;  // lanes per row on the CSR coarse levels

// Vector loads of the coarse sweeps: the read-only path for vectors written by earlier launches,
// the L2 path for vectors written earlier in the same launch (the cluster tail below).
struct LdRO {
  template <class T>
  __device__ __forceinline__ double operator()(const T* p) const { return (double)__ldg(p); }
};
struct LdL2 {
  template <class T>
  __device__ __forceinline__ double operator()(const T* p) const { return (double)__ldcg(p); }
};

// Coarse levels (CSR): G consecutive lanes share one row, each lane takes every G-th entry, and
// the partial sums meet through warp shuffles.  Coarse rows are long and there are few of them,
// so splitting rows keeps enough loads in flight.  The warp-level loop bound keeps every lane of
// a warp in the shuffles.  The row sweeps are device functions over (warp, nWarps) so that the
// per-level kernels and the cluster tail run the same arithmetic.
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, G);
  return v;
}

// Down, part 1 on a CSR level: x = w D^-1 b, x2 = b - A x.
template <int G, class T, class LD>
__device__ __forceinline__ void resid_csr_rows(const AmgLevelDevT<T>& f, int warp, int nWarps, LD ldv) {
  const int lane = threadIdx.x & 31, sub = lane % G;
  const int rowsPerWarp = 32 / G;
  for (int base = warp * rowsPerWarp; base < f.n; base += nWarps * rowsPerWarp) {
    const int i = base + lane / G;
    double acc = 0.0;
    if (i < f.n) {
      const int k1 = __ldg(&f.rowOff[i + 1]);
      for (int k = __ldg(&f.rowOff[i]) + sub; k < k1; k += G) {
        const int j = __ldg(&f.col[k]);
        acc += ld(&f.val[k]) * (ld(&f.wdinv[j]) * ldv(&f.b[j]));
      }
    }
    acc = group_sum<G>(acc);
    if (i < f.n && sub == 0) {
      const double di = ld(&f.diag[i]), bi = ldv(&f.b[i]);
      const double xi = ld(&f.wdinv[i]) * bi;
      f.x[i] = (T)xi;
      f.x2[i] = (T)(bi - di * xi - acc);
    }
  }
}

// Down on a CSR level in one sweep: warp per aggregate I of the next level, its member rows G
// lanes each (32/G at a time); x = w D^-1 b for every member and b_next[I] = the sum over the
// members, in member order, of their T-rounded residuals b - A x.  These are the values of
// resid_csr_rows followed by restrict_rows without the round trip of r through memory and with
// one launch instead of two; an aggregate's members run one after another, so the sweep pays off
// on the small levels only (kFusedDownRows).
template <int G, class T, class LD>
__device__ __forceinline__ void down_csr_aggs(const AmgLevelDevT<T>& f, T* bNext, int warp, int nWarps, LD ldv) {
  const int lane = threadIdx.x & 31, sub = lane % G, grp = lane / G;
  constexpr int NG = 32 / G;
  for (int I = warp; I < f.nc; I += nWarps) {
    const int m0 = __ldg(&f.memOff[I]), m1 = __ldg(&f.memOff[I + 1]);
    double sum = 0.0;
    for (int mb = m0; mb < m1; mb += NG) {
      const int mm = mb + grp;
      double acc = 0.0;
      int i = 0;
      if (mm < m1) {
        i = __ldg(&f.mem[mm]);
        const int2 kr = __ldg(&f.memRow[mm]);
        const int k1 = kr.y;
        for (int k = kr.x + sub; k < k1; k += G) {
          const int j = __ldg(&f.col[k]);
          acc += ld(&f.val[k]) * (ld(&f.wdinv[j]) * ldv(&f.b[j]));
        }
      }
      acc = group_sum<G>(acc);
      double r = 0.0;
      if (mm < m1 && sub == 0) {
        const double di = ld(&f.diag[i]), bi = ldv(&f.b[i]);
        const double xi = ld(&f.wdinv[i]) * bi;
        f.x[i] = (T)xi;
        r = (double)(T)(bi - di * xi - acc);
      }
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        const double rg = __shfl_sync(0xffffffffu, r, g * G);
        if (mb + g < m1) sum += rg;
      }
    }
    if (lane == 0) bNext[I] = (T)sum;
  }
}

// Up on a CSR level: out = xt + w D^-1 (b - A xt) with xt = x + corr e[agg].
template <int G, class T, class LD>
__device__ __forceinline__ void up_csr_rows(const AmgLevelDevT<T>& f, const T* e, double corr, T* out, int warp,
                                            int nWarps, LD ldv) {
  const int lane = threadIdx.x & 31, sub = lane % G;
  const int rowsPerWarp = 32 / G;
  for (int base = warp * rowsPerWarp; base < f.n; base += nWarps * rowsPerWarp) {
    const int i = base + lane / G;
    double acc = 0.0;
    if (i < f.n) {
      const int k1 = __ldg(&f.rowOff[i + 1]);
      for (int k = __ldg(&f.rowOff[i]) + sub; k < k1; k += G) {
        const int j = __ldg(&f.col[k]);
        acc += ld(&f.val[k]) * (ldv(&f.x[j]) + corr * ldv(&e[__ldg(&f.colAgg[k])]));
      }
    }
    acc = group_sum<G>(acc);
    if (i < f.n && sub == 0) {
      const double di = ld(&f.diag[i]);
      const double xi = ldv(&f.x[i]) + corr * ldv(&e[__ldg(&f.agg[i])]);
      out[i] = (T)(xi + ld(&f.wdinv[i]) * (ldv(&f.b[i]) - di * xi - acc));
    }
  }
}

// Down, part 2: piecewise-constant restriction b_next[I] = sum of r over the rows of I
// (thread t of nT).
template <class T, class LD>
__device__ __forceinline__ void restrict_rows(const AmgLevelDevT<T>& f, T* bNext, int t, int nT, LD ldv) {
  for (int I = t; I < f.nc; I += nT) {
    double acc = 0.0;
    const int m1 = __ldg(&f.memOff[I + 1]);
#pragma unroll 4
    for (int mm = __ldg(&f.memOff[I]); mm < m1; ++mm) acc += ldv(&f.x2[__ldg(&f.mem[mm])]);
    bNext[I] = (T)acc;
  }
}

// Coarsest level: x = A^-1 b with the stored dense inverse (double), warp per row, lanes across
// the row (coalesced).
template <class T, class LD>
__device__ __forceinline__ void dense_rows(int n, const double* inv, const T* b, T* x, int warp, int nWarps, LD ldv) {
  const int lane = threadIdx.x & 31;
  for (int i = warp; i < n; i += nWarps) {
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += __ldg(&inv[(size_t)i * n + j]) * ldv(&b[j]);
    s = warp_sum(s);
    if (lane == 0) x[i] = (T)s;
  }
}

template <int G, class T>
__global__ void __launch_bounds__(kBlock) k_amg_resid_csr(const int* done, AmgLevelDevT<T> f, double omega) {
  if (*done) return;
  resid_csr_rows<G>(f, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, (gridDim.x * blockDim.x) >> 5, LdRO{});
}

template <int G, class T>
__global__ void __launch_bounds__(kBlock) k_amg_down_csr(const int* done, AmgLevelDevT<T> f, T* bNext) {
  if (*done) return;
  down_csr_aggs<G>(f, bNext, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, (gridDim.x * blockDim.x) >> 5, LdRO{});
}

template <int G, class T>
__global__ void __launch_bounds__(kBlock) k_amg_up_csr(const int* done, AmgLevelDevT<T> f, const T* e, double omega,
                                                       double corr, T* out) {
  if (*done) return;
  up_csr_rows<G>(f, e, corr, out, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, (gridDim.x * blockDim.x) >> 5,
                 LdRO{});
}

template <class T>
__global__ void __launch_bounds__(kBlock) k_amg_restrict(const int* done, AmgLevelDevT<T> f, T* bNext) {
  if (*done) return;
  restrict_rows(f, bNext, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, LdRO{});
}

// Up: prolongate the coarse correction and post-smooth (one weighted-Jacobi sweep) in one pass:
// xt_j = x_j + corr * e[agg(j)] on the fly, out_i = xt_i + w D^-1 (b_i - (A xt)_i).
// On level 0 it also forms r.z for the PCG recurrence.
template <class T, int WM>
__global__ void __launch_bounds__(kBlock) k_amg_up(const int* doneFlag, AmgLevelDevT<T> f, const T* e, double omega,
                                                   double corr, T* out, int finest, PcgArgsT<T> a) {
  __shared__ double sm[32];
  if (*doneFlag) return;
  double acc[1] = {0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < f.n; i += gridDim.x * blockDim.x) {
    const double di = ld(&f.diag[i]);
    const double xi = ld(&f.x[i]) + corr * ld(&e[__ldg(&f.agg[i])]);
    double ax = di * xi;
    if constexpr (WM == 0) {
      const int s = i >> 5;
      const int b = __ldg(&f.sliceOff[s]) + (i & 31);
      const int W = (__ldg(&f.sliceOff[s + 1]) - __ldg(&f.sliceOff[s])) >> 5;
      // unrolled so the col -> agg -> e load chains of several entries are in flight together
#pragma unroll 4
      for (int k = 0; k < W; ++k) {
        const int ee = b + (k << 5);
        const int j = __ldg(&f.col[ee]);
        ax += ld(&f.val[ee]) * (ld(&f.x[j]) + corr * ld(&e[__ldg(&f.agg[j])]));
      }
    } else {
      int c[WM];
      double v[WM];
      sell_regs<WM>(f.sliceOff, f.col, f.val, i, c, v);
      int g[WM];
#pragma unroll
      for (int k = 0; k < WM; ++k) g[k] = __ldg(&f.agg[c[k]]);
#pragma unroll
      for (int k = 0; k < WM; ++k) ax += v[k] * (ld(&f.x[c[k]]) + corr * ld(&e[g[k]]));
    }
    const double bi = (double)f.b[i];
    const T xn = (T)(xi + ld(&f.wdinv[i]) * (bi - ax));
    out[i] = xn;
    if (finest) acc[0] += bi * (double)xn;
  }
  if (!finest || a.mode != 0) return;
  if (grid_reduce<1>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    const double rzOld = a.sc[0];
    a.sc[2] = a.fl[3] ? 0.0 : acc[0] / rzOld;
    a.sc[0] = acc[0];
  }
}

// Coarsest level on its own: one block.
template <class T>
__global__ void k_amg_dense_apply(const int* done, int n, const double* inv, const T* b, T* x) {
  if (*done) return;
  dense_rows(n, inv, b, x, threadIdx.x >> 5, blockDim.x >> 5, LdRO{});
}

// The coarse tail of the V-cycle in one launch: levels lv[0..nLev-2] (CSR) down, the dense
// level lv[nLev-1], and the same levels up, on one thread-block cluster whose barriers order the
// sweeps.  Every sweep is the per-level kernels' arithmetic; vectors written inside the launch
// are read through L2.  All CTAs of the cluster take the same barriers (the loop bounds and the
// done flag are uniform), so each barrier completes.
constexpr int kTailThreads = 1024;
constexpr int kTailMaxLevels = 12;
template <class T>
struct AmgTailArgs {
  int nLev;
  AmgLevelDevT<T> lv[kTailMaxLevels];
  const double* dense;
  double corr;
};

template <class T>
__global__ void __launch_bounds__(kTailThreads, 1) k_amg_tail(const int* done, const __grid_constant__ AmgTailArgs<T> a) {
  if (*done) return;
  cg::cluster_group cl = cg::this_cluster();
  const int t = (int)cl.block_rank() * blockDim.x + threadIdx.x;
  const int nT = (int)cl.num_blocks() * blockDim.x;
  const int warp = t >> 5, nWarps = nT >> 5;
  const int L = a.nLev;
  for (int l = 0; l + 1 < L; ++l) {
    resid_csr_rows<kCoarseLanes>(a.lv[l], warp, nWarps, LdL2{});
    cl.sync();
    restrict_rows(a.lv[l], a.lv[l + 1].b, t, nT, LdL2{});
    cl.sync();
  }
  dense_rows(a.lv[L - 1].n, a.dense, a.lv[L - 1].b, a.lv[L - 1].x, warp, nWarps, LdL2{});
  for (int l = L - 2; l >= 0; --l) {
    cl.sync();
    const T* e = (l + 1 == L - 1) ? a.lv[l + 1].x : a.lv[l + 1].x2;
    up_csr_rows<kCoarseLanes>(a.lv[l], e, a.corr, a.lv[l].x2, warp, nWarps, LdL2{});
  }
}

// Galerkin values of the next level: one gather list per coarse storage entry (sums in double).
template <class T>
__global__ void __launch_bounds__(kBlock) k_amg_galerkin(AmgLevelDevT<T> f, T* valNext, T* diagNext, T* wdinvNext,
                                                         double omega) {
  const int nT = f.nEntNext + f.nc;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nT; t += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = f.gOff[t]; k < f.gOff[t + 1]; ++k) {
      const int idx = f.gIdx[k];
      s += idx >= 0 ? (double)f.val[idx] : (double)f.diag[-1 - idx];
    }
    if (t < f.nEntNext) {
      valNext[t] = (T)s;
    } else {
      diagNext[t - f.nEntNext] = (T)s;
      wdinvNext[t - f.nEntNext] = (T)(omega / s);
    }
  }
}

// Dense inverse of the coarsest matrix by in-place Gauss-Jordan in double (SPD, no pivoting
// needed); a pivot below 1e-13 of the largest diagonal (singular, all-Neumann systems) gets a
// zero row/column, i.e. the correction ignores the null direction.  One block of 32 warps: the
// matrix is assembled in shared memory, then held in registers, warp w owning rows w, w+32, ...
// and lane l columns l, l+32, ... (NC chunks each, n <= 32 NC).  A pivot step is one barrier:
// the warp owning row k broadcasts the pivot by shuffle and publishes the scaled row, the lanes
// owning column k publish the old column (double-buffered), and every thread updates its entries.
// Per entry the arithmetic is the textbook step: row k / piv, A_kk = 1 / piv,
// A_ij -= A_ik (A_kj / piv), A_ik = -A_ik / piv.
constexpr int kDenseMax = 160;  // largest coarsest level (rows)

template <class T, int NC>
__global__ void __launch_bounds__(1024, 1) k_amg_dense_factor(AmgLevelDevT<T> c, double* inv) {
  extern __shared__ double A[];
  __shared__ double rowk[2][kDenseMax], colk[2][kDenseMax];
  __shared__ int skipk[2];
  __shared__ double dmax;
  const int n = c.n;
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) A[t] = 0.0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {  // the coarsest level is always CSR
    A[i * n + i] = (double)c.diag[i];
    for (int k = c.rowOff[i]; k < c.rowOff[i + 1]; ++k) {
      const int j = c.col[k];
      if (j != i) A[i * n + j] += (double)c.val[k];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0.0;
    for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(A[i * n + i]));
    dmax = mx;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double a[NC][NC];
#pragma unroll
  for (int p = 0; p < NC; ++p)
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      const int i = w + 32 * p, j = lane + 32 * q;
      a[p][q] = (i < n && j < n) ? A[i * n + j] : 0.0;
    }
  __syncthreads();
  const double dm = dmax;
  // pivot k = 32 kc + kw: the chunk kc is a compile-time index, so every register access is static
#pragma unroll
  for (int kc = 0; kc < NC; ++kc) {
    for (int kw = 0; kw < 32; ++kw) {
      const int k = 32 * kc + kw;
      if (k >= n) break;  // uniform over the block
      const int buf = k & 1;
      if (w == kw) {  // row k: pivot by shuffle from lane kw, scaled row to shared memory
        const double piv = __shfl_sync(0xffffffffu, a[kc][kc], kw);
        if (lane == 0) skipk[buf] = fabs(piv) <= 1e-13 * dm;
#pragma unroll
        for (int q = 0; q < NC; ++q) {
          const int j = lane + 32 * q;
          if (j < n) rowk[buf][j] = j == k ? 1.0 / piv : a[kc][q] / piv;
        }
      }
      if (lane == kw) {  // column k before the step
#pragma unroll
        for (int p = 0; p < NC; ++p) {
          const int i = w + 32 * p;
          if (i < n) colk[buf][i] = a[p][kc];
        }
      }
      __syncthreads();
      // every entry takes the rank-1 update, then column k and row k (in that order) are
      // overwritten by their owners; entries past n stay zero and are never stored
      if (skipk[buf] == 0) {
        double rk[NC], ck[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) rk[q] = lane + 32 * q < n ? rowk[buf][lane + 32 * q] : 0.0;
#pragma unroll
        for (int p = 0; p < NC; ++p) ck[p] = w + 32 * p < n ? colk[buf][w + 32 * p] : 0.0;
#pragma unroll
        for (int p = 0; p < NC; ++p)
#pragma unroll
          for (int q = 0; q < NC; ++q) a[p][q] -= ck[p] * rk[q];
        if (lane == kw) {
          const double rkk = rowk[buf][k];
#pragma unroll
          for (int p = 0; p < NC; ++p) a[p][kc] = -ck[p] * rkk;
        }
        if (w == kw) {
#pragma unroll
          for (int q = 0; q < NC; ++q) a[kc][q] = rk[q];
        }
      } else {
        if (lane == kw) {
#pragma unroll
          for (int p = 0; p < NC; ++p) a[p][kc] = 0.0;
        }
        if (w == kw) {
#pragma unroll
          for (int q = 0; q < NC; ++q) a[kc][q] = 0.0;
        }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < NC; ++p)
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      const int i = w + 32 * p, j = lane + 32 * q;
      if (i < n && j < n) inv[(size_t)i * n + j] = a[p][q];
    }
}

// ---------------------------------------------------------------- mixed-precision defect
// r = b - A x in double (float matrix, double x), r32 = r; per component |r|^2, |b|^2.
__global__ void __launch_bounds__(kBlock) k_defect(DefectArgs a) {
  __shared__ double sm[6 * 32];
  const int n = a.A.n;
  bool act[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) act[c] = c < a.nc && !(a.frozen && a.frozen[c]);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) continue;
      const size_t o = (size_t)c * n;
      const double bb = a.b[o + r];
      const double rr = bb - sell_row(a.A, r, a.x + o);
      a.r32[o + r] = (float)rr;
      acc[2 * c] += rr * rr;
      acc[2 * c + 1] += bb * bb;
    }
  }
  if (grid_reduce<6>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    _Pragma("unroll") for (int c = 0; c < 3; ++c) if (c < a.nc) {
      if (!act[c]) {
        a.fl[4 * c] = 1;
        continue;
      }
      a.sc[8 * c] = acc[2 * c];
      a.sc[8 * c + 1] = acc[2 * c + 1];
      a.fl[4 * c] = sqrt(acc[2 * c]) <= fmax(a.atol, a.rtol * sqrt(acc[2 * c + 1])) ? 1 : 0;
    }
  }
}

// wdinv = omega / diag (weighted-Jacobi smoother weights of a level-0 matrix)
__global__ void __launch_bounds__(kBlock) k_jacobi_weights(int n, double omega, const double* diag, double* wdinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) wdinv[i] = omega / diag[i];
}

__global__ void __launch_bounds__(kBlock) k_apply_correction(size_t n, double* x, float* dx) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    x[i] += (double)dx[i];
    dx[i] = 0.0f;
  }
}

}  // namespace

template <class T>
void bicg_init(const LaunchCfg& lc, const BicgArgsT<T>& a) {
  g_launches += 1;
  with_width(a.A.maxW, [&](auto W) { launch_rows(lc, lc.rowBlocks, k_bicg_init<T, W.value>, a); });
}
// One BiCGSTAB iteration; apply (when given) is the right preconditioner of the active
// components after the p and the s updates (the vector kernels then leave ph and sh to it).
template <class T>
static void bicg_step(const LaunchCfg& lc, const BicgArgsT<T>& a, void (*apply)(void*, int, int), void* ctx) {
  const double vbytes = lc.ab ? lc.ab->bicg_spmv(a.nc) * (sizeof(T) == 4 ? 0.5 : 1.0) : 0.0;
  {
    ProfScope ps(lc, kKfBicgVector, 0.0);
    k_bicg_p<T><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
  }
  if (apply)
    for (int c = 0; c < a.nc; ++c) apply(ctx, c, 0);
  {
    ProfScope ps(lc, kKfBicgSpmv, vbytes);
    with_width(a.A.maxW, [&](auto W) { launch_rows(lc, lc.rowBlocks, k_bicg_v<T, W.value>, a); });
  }
  {
    ProfScope ps(lc, kKfBicgVector, 0.0);
    k_bicg_s<T><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
  }
  if (apply)
    for (int c = 0; c < a.nc; ++c) apply(ctx, c, 1);
  {
    ProfScope ps(lc, kKfBicgSpmv, vbytes);
    with_width(a.A.maxW, [&](auto W) { launch_rows(lc, lc.rowBlocks, k_bicg_t<T, W.value>, a); });
  }
  {
    ProfScope ps(lc, kKfBicgVector, 0.0);
    launch_rows(lc, lc.rowBlocks, k_bicg_x<T>, a);
  }
}
template <class T>
void bicg_iteration(const LaunchCfg& lc, const BicgArgsT<T>& a) {
  bicg_step(lc, a, nullptr, nullptr);
}
template <class T>
void bicg_iteration_precond(const LaunchCfg& lc, const BicgArgsT<T>& a, void (*apply)(void*, int, int), void* ctx) {
  bicg_step(lc, a, apply, ctx);
}

template <class T>
void pcg_init(const LaunchCfg& lc, const PcgArgsT<T>& a) {
  g_launches += 1;
  with_width(a.A.maxW, [&](auto W) { launch_rows(lc, lc.rowBlocks, k_pcg_init<T, W.value>, a); });
}

static int blocks_for(int n, int cap) { return std::max(1, std::min(cap, (n + kBlock - 1) / kBlock)); }

// First level of the cluster tail; L - 1 (the dense level alone, no tail) when the tail is off or
// no CSR level is small enough.  Level sizes fall with depth, so the tail is a suffix.
template <class T>
static int tail_start(const AmgDevT<T>* amg) {
  const int L = amg->nLevels;
  if (amg->tailCluster <= 0 || amg->tailRows <= 0) return L - 1;
  int t0 = L - 1;
  while (t0 - 1 >= 1 && amg->lv[t0 - 1].n <= amg->tailRows && !amg->lv[t0 - 1].sliceOff &&
         L - (t0 - 1) <= kTailMaxLevels)
    --t0;
  return t0;
}

static cudaLaunchConfig_t tail_config(cudaStream_t s, int cluster, cudaLaunchAttribute* at) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(cluster);
  cfg.blockDim = dim3(kTailThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cluster;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

template <class T>
static void launch_tail(const LaunchCfg& lc, const int* done, const AmgDevT<T>* amg, int t0) {
  AmgTailArgs<T> ta{};
  ta.nLev = amg->nLevels - t0;
  for (int l = 0; l < ta.nLev; ++l) ta.lv[l] = amg->lv[t0 + l];
  ta.dense = amg->dense;
  ta.corr = amg->corr;
  cudaLaunchAttribute at[1];
  const cudaLaunchConfig_t cfg = tail_config(lc.stream, amg->tailCluster, at);
  cudaLaunchKernelEx(&cfg, k_amg_tail<T>, done, ta);
}

// Cluster size of the tail: 16 CTAs (a non-portable size) when the device can co-schedule them,
// else 8; 0 (no tail) when neither fits.
template <class T>
void amg_configure_tail(AmgDevT<T>& amg, int tailRows, cudaStream_t s) {
  amg.tailRows = tailRows;
  amg.tailCluster = 0;
  if (tailRows <= 0) return;
  cudaFuncSetAttribute(k_amg_tail<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  for (int cs : {16, 8}) {
    cudaLaunchAttribute at[1];
    const cudaLaunchConfig_t cfg = tail_config(s, cs, at);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_amg_tail<T>, &cfg) == cudaSuccess && n > 0) {
      amg.tailCluster = cs;
      return;
    }
    cudaGetLastError();
  }
}

// One V-cycle z = M^-1 r_new, fused at level 0 with the PCG update r_new = r - alpha q,
// x += alpha p (see k_amg_resid0): variant v reads the residual buffer v (0: a.r, 1: a.r2), writes
// the other and updates x with p_v.
template <class T>
static void vcycle(const LaunchCfg& lc, const PcgArgsT<T>& a, const AmgDevT<T>* amg, int v) {
  const int L = amg->nLevels;
  const T* rIn = v ? a.r2 : a.r;
  T* rOut = v ? a.r : a.r2;
  const T* p = v ? a.p1 : a.p0;
  AmgLevelDevT<T> f0 = amg->lv[0];
  f0.b = rOut;  // level 0 right-hand side is the new PCG residual
  {
    const AmgLevelDevT<T>& f = f0;
    ProfScope ps(lc, kKfAmgResid0, 0.0, 2);
    const int nb = blocks_for(f.n, lc.rowBlocks);
    with_width(f.maxW, [&](auto W) { launch_rows(lc, nb, k_amg_resid0<T, W.value>, a, f, rIn, rOut, p); });
    k_amg_restrict<T><<<blocks_for(f.nc, lc.rowBlocks), kBlock, 0, lc.stream>>>(a.fl, f, amg->lv[1].b);
  }
  {
    const int t0 = tail_start(amg);
    auto fused = [&](const AmgLevelDevT<T>& f) { return !f.sliceOff && f.n <= amg->fusedDownRows; };
    int nl = 1;
    for (int l = 1; l < t0; ++l) nl += fused(amg->lv[l]) ? 2 : 3;
    ProfScope ps(lc, kKfAmgCoarse, 0.0, nl);
    for (int l = 1; l < t0; ++l) {
      const AmgLevelDevT<T>& f = amg->lv[l];
      if (f.sliceOff) {  // large coarse level in SELL-32: the level-0 kernels, thread per row
        const int nb = blocks_for(f.n, lc.rowBlocks);
        with_width(f.maxW, [&](auto W) { launch_rows(lc, nb, k_amg_resid<T, W.value>, a.fl, f, amg->omega); });
        k_amg_restrict<T><<<blocks_for(f.nc, lc.rowBlocks), kBlock, 0, lc.stream>>>(a.fl, f, amg->lv[l + 1].b);
        continue;
      }
      if (fused(f)) {
        k_amg_down_csr<kCoarseLanes, T><<<blocks_for(f.nc * 32, lc.rowBlocks), kBlock, 0, lc.stream>>>(
            a.fl, f, amg->lv[l + 1].b);
        continue;
      }
      k_amg_resid_csr<kCoarseLanes, T><<<blocks_for(f.n * kCoarseLanes, lc.rowBlocks), kBlock, 0, lc.stream>>>(
          a.fl, f, amg->omega);
      k_amg_restrict<T><<<blocks_for(f.nc, lc.rowBlocks), kBlock, 0, lc.stream>>>(a.fl, f, amg->lv[l + 1].b);
    }
    if (t0 < L - 1) {
      launch_tail(lc, a.fl, amg, t0);
    } else {
      const AmgLevelDevT<T>& c = amg->lv[L - 1];
      k_amg_dense_apply<T><<<1, 1024, 0, lc.stream>>>(a.fl, c.n, amg->dense, c.b, c.x);
    }
    for (int l = t0 - 1; l >= 1; --l) {
      const AmgLevelDevT<T>& f = amg->lv[l];
      // correction from the coarser level: its smoothed solution (x2), or x on the coarsest
      const T* e = (l + 1 == L - 1) ? amg->lv[l + 1].x : amg->lv[l + 1].x2;
      if (f.sliceOff) {
        const int nb = blocks_for(f.n, lc.rowBlocks);
        with_width(f.maxW, [&](auto W) {
          launch_rows(lc, nb, k_amg_up<T, W.value>, a.fl, f, e, amg->omega, amg->corr, f.x2, 0, a);
        });
        continue;
      }
      k_amg_up_csr<kCoarseLanes, T><<<blocks_for(f.n * kCoarseLanes, lc.rowBlocks), kBlock, 0, lc.stream>>>(
          a.fl, f, e, amg->omega, amg->corr, f.x2);
    }
  }
  {
    const AmgLevelDevT<T>& f = f0;
    const T* e = (L == 2) ? amg->lv[1].x : amg->lv[1].x2;
    ProfScope ps(lc, kKfAmgUp0, 0.0);
    const int nb = blocks_for(f.n, lc.rowBlocks);
    with_width(f.maxW, [&](auto W) {
      launch_rows(lc, nb, k_amg_up<T, W.value>, a.fl, f, e, amg->omega, amg->corr, a.z, 1, a);
    });
  }
}

// V-cycle variant v (graph when captured)
template <class T>
static void apply_vcycle(const LaunchCfg& lc, const PcgArgsT<T>& a, const AmgDevT<T>* amg, int v) {
  if (amg->graph[v]) {
    g_launches += amg->graphKernels;
    cudaGraphLaunch(amg->graph[v], lc.stream);
  } else {
    vcycle(lc, a, amg, v);
  }
}

template <class T>
void pcg_precondition(const LaunchCfg& lc, const PcgArgsT<T>& a, const AmgDevT<T>* amg) {
  if (!amg || amg->nLevels < 2) {
    g_launches += 1;
    k_pcg_jacobi<T><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
  } else {
    apply_vcycle(lc, a, amg, 0);  // right after pcg_init: no update, r copied to r2
  }
}

// Records the two V-cycle variants into CUDA graphs.  Every pointer and scalar the V-cycle kernels
// read is fixed for the life of the hierarchy (values change on refresh, addresses do not; the
// callers keep x, r, r2, p0, p1, q and z at fixed addresses), so the graphs are captured once and
// replayed for every preconditioner application.
template <class T>
static cudaError_t pcg_capture_loop(const LaunchCfg& lc, const PcgArgsT<T>& a, AmgDevT<T>& amg);

// ANB_NO_LOOP_GRAPH=1 keeps the solver loops on the host (for measurements)
static bool loop_graphs_off() {
  const char* s = std::getenv("ANB_NO_LOOP_GRAPH");
  return s && s[0] == '1';
}

template <class T>
cudaError_t amg_capture_graph(const LaunchCfg& lc, const PcgArgsT<T>& a, AmgDevT<T>& amg) {
  amg_release_graphs(amg);
  LaunchCfg quiet = lc;
  quiet.prof = nullptr;
  for (int v = 0; v < 2; ++v) {
    const long long before = g_launches.load();
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(lc.stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    vcycle(quiet, a, &amg, v);
    e = cudaStreamEndCapture(lc.stream, &g);
    amg.graphKernels = (int)(g_launches.load() - before);
    g_launches -= amg.graphKernels;
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&amg.graph[v], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return e;
  }
  if (a.mode == 0 && !loop_graphs_off()) pcg_capture_loop(lc, a, amg);  // else the host loop runs
  return cudaSuccess;
}

// p = z + beta p_old, q = A p of iteration `it` (p0/p1 alternate)
template <class T>
static void launch_pq(const LaunchCfg& lc, const PcgArgsT<T>& a, int it) {
  const T* pOld = (it & 1) ? a.p1 : a.p0;
  T* pNew = (it & 1) ? a.p0 : a.p1;
  // algorithmic bytes: 12 B per off-diagonal (value + column) and 40 B per row in FP64; values
  // and vectors halve in FP32
  const double by = lc.ab ? (sizeof(T) == 8 ? lc.ab->pcg_spmv() : 20.0 * lc.ab->C + 8.0 * lc.ab->nnzOff) : 0.0;
  ProfScope ps(lc, kKfPcgSpmv, by);
  with_width(a.A.maxW, [&](auto W) { launch_rows(lc, lc.rowBlocks, k_pcg_pq<T, W.value>, a, pOld, pNew); });
}

// A solver loop as one graph: cond(h) (a one-thread kernel that sets the condition h), then a
// while node whose body is body() followed by cond(h) again.  Launches recorded by body() are not
// counted in g_launches.  On failure *out is null and the error state is cleared.
template <class Body, class Cond>
static cudaError_t capture_while(cudaStream_t s, Body&& body, Cond&& cond, cudaGraphExec_t* out) {
  *out = nullptr;
  const long long before = g_launches.load();
  cudaGraph_t g = nullptr, bodyGraph = nullptr;
  cudaGraphConditionalHandle h{};
  cudaGraphNode_t pre = nullptr, loop = nullptr;
  size_t nPre = 1;
  cudaGraphNodeParams np{};
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(s, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cond(h);
    e = cudaStreamEndCapture(s, &g);
  }
  if (e == cudaSuccess) e = cudaGraphGetNodes(g, &pre, &nPre);
  if (e == cudaSuccess && nPre != 1) e = cudaErrorInvalidValue;
  if (e == cudaSuccess) {
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    e = cudaGraphAddNode(&loop, g, &pre, 1, &np);
  }
  if (e == cudaSuccess) {
    bodyGraph = np.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(s, bodyGraph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  }
  if (e == cudaSuccess) {
    body();
    cond(h);
    e = cudaStreamEndCapture(s, &bodyGraph);
  }
  g_launches = before;
  if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    *out = nullptr;
    cudaGetLastError();
  }
  return e;
}

// The PCG iterations of a solve as one graph (capture_while): the body is two AMG-PCG iterations
// (even: p0 -> p1 with V-cycle variant 1; odd: p1 -> p0 with variant 0).  The condition stays set
// while the solve is not done, for at most maxit / 2 + 3 evaluations; iterations after
// convergence return at once, as in the host loop.  The kernels are those of pcg_iteration with
// the same arguments, so the iterates are the same bit for bit.
template <class T>
static cudaError_t pcg_capture_loop(const LaunchCfg& lc, const PcgArgsT<T>& a, AmgDevT<T>& amg) {
  if (amg.loop) cudaGraphExecDestroy(amg.loop);
  amg.loop = nullptr;
  LaunchCfg quiet = lc;
  quiet.prof = nullptr;
  const int maxTrips = a.maxit / 2 + 3;
  const cudaError_t e = capture_while(
      lc.stream,
      [&] {
        for (int it = 0; it < 2; ++it) {
          launch_pq(quiet, a, it);
          vcycle(quiet, a, &amg, (it + 1) & 1);
        }
      },
      [&](cudaGraphConditionalHandle h) { k_pcg_loop_cond<<<1, 1, 0, lc.stream>>>(h, a.fl, maxTrips); },
      &amg.loop);
  if (e == cudaSuccess) amg.loopArgs = a;
  return e;
}

template <class T>
static bool same_pcg_buffers(const PcgArgsT<T>& x, const PcgArgsT<T>& y) {
  return x.A.val == y.A.val && x.A.diag == y.A.diag && x.A.col == y.A.col && x.x == y.x && x.r == y.r &&
         x.r2 == y.r2 && x.z == y.z && x.p0 == y.p0 && x.p1 == y.p1 && x.q == y.q && x.sc == y.sc &&
         x.fl == y.fl && x.maxit == y.maxit && x.mode == y.mode && x.red.partials == y.red.partials;
}

template <class T>
bool pcg_loop_launch(const LaunchCfg& lc, const PcgArgsT<T>& a, const AmgDevT<T>& amg) {
  if (!amg.loop || !same_pcg_buffers(a, amg.loopArgs)) return false;
  return cudaGraphLaunch(amg.loop, lc.stream) == cudaSuccess;
}

template <class T>
void amg_release_graphs(AmgDevT<T>& amg) {
  for (auto& g : amg.graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
  if (amg.loop) cudaGraphExecDestroy(amg.loop);
  amg.loop = nullptr;
  amg.graphKernels = 0;
}

template <class T>
static bool same_bicg_buffers(const BicgArgsT<T>& x, const BicgArgsT<T>& y) {
  return x.A.val == y.A.val && x.A.diag == y.A.diag && x.A.col == y.A.col && x.nc == y.nc && x.x == y.x &&
         x.r == y.r && x.rh == y.rh && x.p == y.p && x.v == y.v && x.s == y.s && x.t == y.t && x.ph == y.ph &&
         x.sh == y.sh && x.sc == y.sc && x.fl == y.fl && x.maxit == y.maxit && x.precond == y.precond &&
         x.red.partials == y.red.partials;
}

// The BiCGSTAB iterations of a solve as one graph (capture_while): two Jacobi-preconditioned
// iterations per trip, the condition set while a component is not done (at most maxit / 2 + 3
// evaluations); the kernels of bicg_iteration with the same arguments.
template <class T>
bool bicg_loop_launch(const LaunchCfg& lc, const BicgArgsT<T>& a, BicgLoopT<T>& loop) {
  if (a.precond || loop.failed || loop_graphs_off()) return false;
  if (loop.exec && !same_bicg_buffers(a, loop.args)) bicg_loop_release(loop);
  if (!loop.exec) {
    LaunchCfg quiet = lc;
    quiet.prof = nullptr;
    const int maxTrips = a.maxit / 2 + 3;
    const cudaError_t e = capture_while(
        lc.stream,
        [&] {
          for (int k = 0; k < 2; ++k) bicg_step(quiet, a, nullptr, nullptr);
        },
        [&](cudaGraphConditionalHandle h) { k_bicg_loop_cond<<<1, 1, 0, lc.stream>>>(h, a.fl, a.nc, maxTrips); },
        &loop.exec);
    if (e != cudaSuccess) {
      loop.failed = true;
      return false;
    }
    loop.args = a;
  }
  return cudaGraphLaunch(loop.exec, lc.stream) == cudaSuccess;
}

template <class T>
void bicg_loop_release(BicgLoopT<T>& loop) {
  if (loop.exec) cudaGraphExecDestroy(loop.exec);
  loop.exec = nullptr;
}

template <class T>
void pcg_iteration(const LaunchCfg& lc, const PcgArgsT<T>& a, int it, const AmgDevT<T>* amg) {
  T* pNew = (it & 1) ? a.p0 : a.p1;
  const bool useAmg = amg && amg->nLevels >= 2;
  launch_pq(lc, a, it);
  if (useAmg) {
    // the V-cycle's level-0 sweep applies x += alpha pNew, r -= alpha q: variant (it + 1) & 1 reads
    // the residual this iteration starts from and uses pNew (p1 on even iterations)
    apply_vcycle(lc, a, amg, (it + 1) & 1);
    return;
  }
  {
    ProfScope ps(lc, kKfPcgUpdate, 0.0);
    k_pcg_xr<T><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a, pNew);
  }
  pcg_precondition(lc, a, amg);
}

template <class T>
void amg_apply(const LaunchCfg& lc, const PcgArgsT<T>& a, const AmgDevT<T>* amg, cudaGraphExec_t* graph) {
  if (graph && !*graph) {
    LaunchCfg quiet = lc;
    quiet.prof = nullptr;
    const long long before = g_launches.load();
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(lc.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      vcycle(quiet, a, amg, 0);
      const cudaError_t e = cudaStreamEndCapture(lc.stream, &g);
      if (e == cudaSuccess && cudaGraphInstantiate(graph, g, 0) != cudaSuccess) *graph = nullptr;
      if (g) cudaGraphDestroy(g);
    }
    g_launches = before;
  }
  if (graph && *graph) {
    g_launches += amg->graphKernels;
    cudaGraphLaunch(*graph, lc.stream);
  } else {
    vcycle(lc, a, amg, 0);
  }
}

template <class T>
void amg_refresh(const LaunchCfg& lc, AmgDevT<T>& amg) {
  for (int l = 0; l + 1 < amg.nLevels; ++l) {
    AmgLevelDevT<T>& f = amg.lv[l];
    AmgLevelDevT<T>& c = amg.lv[l + 1];
    g_launches += 1;
    k_amg_galerkin<T><<<blocks_for(f.nEntNext + f.nc, lc.rowBlocks), kBlock, 0, lc.stream>>>(f, c.val, c.diag,
                                                                                             c.wdinv, amg.omega);
  }
  const AmgLevelDevT<T>& c = amg.lv[amg.nLevels - 1];
  const size_t smem = sizeof(double) * (size_t)c.n * c.n;
  g_launches += 1;
  const int nc = (c.n + 31) / 32;
  auto go = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    kern<<<1, 1024, smem, lc.stream>>>(c, amg.dense);
  };
  if (nc <= 1) go(k_amg_dense_factor<T, 1>);
  else if (nc == 2) go(k_amg_dense_factor<T, 2>);
  else if (nc == 3) go(k_amg_dense_factor<T, 3>);
  else if (nc == 4) go(k_amg_dense_factor<T, 4>);
  else go(k_amg_dense_factor<T, 5>);
}

void launch_defect(const LaunchCfg& lc, const DefectArgs& a) {
  g_launches += 1;
  k_defect<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
}

void launch_jacobi_weights(const LaunchCfg& lc, int n, double omega, const double* diag, double* wdinv) {
  g_launches += 1;
  k_jacobi_weights<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(n, omega, diag, wdinv);
}

void launch_apply_correction(const LaunchCfg& lc, int n, int nc, double* x, float* dx) {
  g_launches += 1;
  k_apply_correction<<<lc.rowBlocks, kBlock, 0, lc.stream>>>((size_t)n * nc, x, dx);
}

#define ANB_INSTANTIATE(T)                                                                    \
  template void bicg_init<T>(const LaunchCfg&, const BicgArgsT<T>&);                          \
  template void bicg_iteration<T>(const LaunchCfg&, const BicgArgsT<T>&);                     \
  template void pcg_init<T>(const LaunchCfg&, const PcgArgsT<T>&);                            \
  template void pcg_iteration<T>(const LaunchCfg&, const PcgArgsT<T>&, int, const AmgDevT<T>*); \
  template void pcg_precondition<T>(const LaunchCfg&, const PcgArgsT<T>&, const AmgDevT<T>*);  \
  template void amg_refresh<T>(const LaunchCfg&, AmgDevT<T>&);                                \
  template cudaError_t amg_capture_graph<T>(const LaunchCfg&, const PcgArgsT<T>&, AmgDevT<T>&);           \
  template bool pcg_loop_launch<T>(const LaunchCfg&, const PcgArgsT<T>&, const AmgDevT<T>&);  \
  template void amg_release_graphs<T>(AmgDevT<T>&);                                           \
  template bool bicg_loop_launch<T>(const LaunchCfg&, const BicgArgsT<T>&, BicgLoopT<T>&);     \
  template void bicg_loop_release<T>(BicgLoopT<T>&);                                          \
  template void amg_configure_tail<T>(AmgDevT<T>&, int, cudaStream_t);                          \
  template void amg_apply<T>(const LaunchCfg&, const PcgArgsT<T>&, const AmgDevT<T>*, cudaGraphExec_t*); \
  template void bicg_iteration_precond<T>(const LaunchCfg&, const BicgArgsT<T>&, void (*)(void*, int, int), void*);
ANB_INSTANTIATE(double)
ANB_INSTANTIATE(float)
#undef ANB_INSTANTIATE

}  // namespace anb
