// Krylov solvers and the aggregation-AMG V-cycle (sm_100a), standing in for the reference's
// HYPRE BiCGSTAB+DiagScale momentum solve (main.cu:2553-2576) and PCG+BoomerAMG pressure solve
// (main.cu:2224-2273, 2617-2676).
//
// All scalars stay on the device: every reduction ends in the last block of its kernel
// (deterministic block-order combination), which also advances the recurrence scalars and the
// convergence flags.  Kernels return immediately once their system is converged, so the host
// can enqueue several iterations between polls without changing the arithmetic.
#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "kernels.cuh"

namespace anb {
namespace {

// y = (D + Off) x for one row of a SELL-32 matrix
__device__ __forceinline__ double sell_row(const DSell& A, int r, const double* x) {
  const int s = r >> 5;
  const int b = __ldg(&A.sliceOff[s]) + (r & 31);
  const int W = (__ldg(&A.sliceOff[s + 1]) - __ldg(&A.sliceOff[s])) >> 5;
  double y = A.diag[r] * x[r];
#pragma unroll 4
  for (int k = 0; k < W; ++k) {
    const int e = b + (k << 5);
    y += __ldg(&A.val[e]) * x[__ldg(&A.col[e])];
  }
  return y;
}

// y_c = (D + Off) x_c for up to three vectors sharing one pass over the matrix row
__device__ __forceinline__ void sell_row3(const DSell& A, int r, const double* x, size_t n, const bool* act, int nc,
                                          double* y) {
  const int s = r >> 5;
  const int b = __ldg(&A.sliceOff[s]) + (r & 31);
  const int W = (__ldg(&A.sliceOff[s + 1]) - __ldg(&A.sliceOff[s])) >> 5;
  const double d = A.diag[r];
  for (int c = 0; c < 3; ++c) y[c] = (c < nc && act[c]) ? d * x[c * n + r] : 0.0;
#pragma unroll 2
  for (int k = 0; k < W; ++k) {
    const int e = b + (k << 5);
    const double v = __ldg(&A.val[e]);
    const int j = __ldg(&A.col[e]);
    for (int c = 0; c < 3; ++c)
      if (c < nc && act[c]) y[c] += v * x[c * n + j];
  }
}

// ---------------------------------------------------------------- BiCGSTAB, nc components
// scalars per component c: sc[8c + 0..7] = rho, rhoN, alpha, omega, eps, rn, -, -
// flags per component c:   fl[4c + 0..3] = done, half, iters, converged

__device__ __forceinline__ bool all_done(const int* fl, int nc) {
  for (int c = 0; c < nc; ++c)
    if (!fl[4 * c]) return false;
  return true;
}

__global__ void __launch_bounds__(kBlock) k_bicg_init(BicgArgs a) {
  __shared__ double sm[6 * 32];
  const int n = a.A.n;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    for (int c = 0; c < a.nc; ++c) {
      const size_t o = (size_t)c * n;
      const double rr = a.b[o + r] - sell_row(a.A, r, a.x + o);
      a.r[o + r] = rr;
      a.rh[o + r] = rr;
      a.p[o + r] = 0.0;
      a.v[o + r] = 0.0;
      acc[2 * c] += rr * rr;
      acc[2 * c + 1] += a.b[o + r] * a.b[o + r];
    }
  }
  if (grid_reduce<6>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    for (int c = 0; c < a.nc; ++c) {
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
  }
}

// p = r + beta (p - omega v); ph = D^-1 p
__global__ void __launch_bounds__(kBlock) k_bicg_p(BicgArgs a) {
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  double beta[3], om[3];
  bool act[3];
  for (int c = 0; c < a.nc; ++c) {
    const double* s = a.sc + 8 * c;
    act[c] = !a.fl[4 * c];
    beta[c] = (s[1] / s[0]) * (s[2] / s[3]);
    om[c] = s[3];
  }
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double dinv = 1.0 / a.A.diag[r];
    for (int c = 0; c < a.nc; ++c) {
      if (!act[c]) continue;
      const size_t i = (size_t)c * n + r;
      const double pn = a.r[i] + beta[c] * (a.p[i] - om[c] * a.v[i]);
      a.p[i] = pn;
      a.ph[i] = dinv * pn;
    }
  }
}

// v = A ph ; alpha = rhoN / (rh . v) ; rho = rhoN
__global__ void __launch_bounds__(kBlock) k_bicg_v(BicgArgs a) {
  __shared__ double sm[3 * 32];
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  bool act[3];
  for (int c = 0; c < a.nc; ++c) act[c] = !a.fl[4 * c];
  double acc[3] = {0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double y[3];
    sell_row3(a.A, r, a.ph, (size_t)n, act, a.nc, y);
    for (int c = 0; c < a.nc; ++c) {
      if (!act[c]) continue;
      const size_t o = (size_t)c * n;
      a.v[o + r] = y[c];
      acc[c] += a.rh[o + r] * y[c];
    }
  }
  if (grid_reduce<3>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    for (int c = 0; c < a.nc; ++c) {
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
__global__ void __launch_bounds__(kBlock) k_bicg_s(BicgArgs a) {
  __shared__ double sm[3 * 32];
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  bool act[3];
  double al[3];
  for (int c = 0; c < a.nc; ++c) {
    act[c] = !a.fl[4 * c];
    al[c] = a.sc[8 * c + 2];
  }
  double acc[3] = {0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double dinv = 1.0 / a.A.diag[r];
    for (int c = 0; c < a.nc; ++c) {
      if (!act[c]) continue;
      const size_t i = (size_t)c * n + r;
      const double sv = a.r[i] - al[c] * a.v[i];
      a.s[i] = sv;
      a.sh[i] = dinv * sv;
      acc[c] += sv * sv;
    }
  }
  if (grid_reduce<3>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    for (int c = 0; c < a.nc; ++c) {
      if (!act[c]) continue;
      if (sqrt(acc[c]) <= a.sc[8 * c + 4]) a.fl[4 * c + 1] = 1;
    }
  }
}

// t = A sh ; omega = (t.s)/(t.t)
__global__ void __launch_bounds__(kBlock) k_bicg_t(BicgArgs a) {
  __shared__ double sm[6 * 32];
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  bool act[3];
  for (int c = 0; c < a.nc; ++c) act[c] = !a.fl[4 * c] && !a.fl[4 * c + 1];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double y[3];
    sell_row3(a.A, r, a.sh, (size_t)n, act, a.nc, y);
    for (int c = 0; c < a.nc; ++c) {
      if (!act[c]) continue;
      const size_t o = (size_t)c * n;
      const double tv = y[c];
      a.t[o + r] = tv;
      acc[2 * c] += tv * a.s[o + r];
      acc[2 * c + 1] += tv * tv;
    }
  }
  if (grid_reduce<6>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    for (int c = 0; c < a.nc; ++c) {
      if (!act[c]) continue;
      a.sc[8 * c + 3] = acc[2 * c + 1] > 0.0 ? acc[2 * c] / acc[2 * c + 1] : 0.0;
    }
  }
}

// x += alpha ph + omega sh ; r = s - omega t ; convergence
__global__ void __launch_bounds__(kBlock) k_bicg_x(BicgArgs a) {
  __shared__ double sm[6 * 32];
  if (all_done(a.fl, a.nc)) return;
  const int n = a.A.n;
  bool act[3], half[3];
  double al[3], om[3];
  for (int c = 0; c < a.nc; ++c) {
    act[c] = !a.fl[4 * c];
    half[c] = a.fl[4 * c + 1] != 0;
    al[c] = a.sc[8 * c + 2];
    om[c] = a.sc[8 * c + 3];
  }
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    for (int c = 0; c < a.nc; ++c) {
      if (!act[c]) continue;
      const size_t i = (size_t)c * n + r;
      if (half[c]) {
        a.x[i] += al[c] * a.ph[i];
      } else {
        a.x[i] += al[c] * a.ph[i] + om[c] * a.sh[i];
        const double rr = a.s[i] - om[c] * a.t[i];
        a.r[i] = rr;
        acc[2 * c] += rr * rr;
        acc[2 * c + 1] += a.rh[i] * rr;
      }
    }
  }
  if (grid_reduce<6>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    for (int c = 0; c < a.nc; ++c) {
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

__global__ void __launch_bounds__(kBlock) k_pcg_init(PcgArgs a) {
  __shared__ double sm[2 * 32];
  const int n = a.A.n;
  double acc[2] = {0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double rr = a.b[r] - sell_row(a.A, r, a.x);
    a.r[r] = rr;
    acc[0] += rr * rr;
    acc[1] += a.b[r] * a.b[r];
  }
  if (grid_reduce<2>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    a.sc[3] = fmax(a.atol, a.rtol * sqrt(acc[1]));
    a.sc[4] = acc[0];
    a.sc[2] = 0.0;
    a.fl[0] = sqrt(acc[0]) <= a.sc[3] ? 1 : 0;
    a.fl[1] = 0;
    a.fl[2] = a.fl[0];
    a.fl[3] = 1;
  }
}

// Jacobi preconditioner z = D^-1 r with rz (used when the AMG is off)
__global__ void __launch_bounds__(kBlock) k_pcg_jacobi(PcgArgs a) {
  __shared__ double sm[32];
  if (a.fl[0]) return;
  const int n = a.A.n;
  double acc[1] = {0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const double z = a.r[r] / a.A.diag[r];
    a.z[r] = z;
    acc[0] += a.r[r] * z;
  }
  if (grid_reduce<1>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    const double rzOld = a.sc[0];
    a.sc[2] = a.fl[3] ? 0.0 : acc[0] / rzOld;
    a.sc[0] = acc[0];
  }
}

// pNew = z + beta pOld (rows and, on the fly, their neighbours); q = A pNew; alpha = rz / (p.q)
__global__ void __launch_bounds__(kBlock) k_pcg_pq(PcgArgs a, const double* pOld, double* pNew) {
  __shared__ double sm[32];
  if (a.fl[0]) return;
  const int n = a.A.n;
  const double beta = a.fl[3] ? 0.0 : a.sc[2];
  double acc[1] = {0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    const int s = r >> 5;
    const int b = __ldg(&a.A.sliceOff[s]) + (r & 31);
    const int W = (__ldg(&a.A.sliceOff[s + 1]) - __ldg(&a.A.sliceOff[s])) >> 5;
    const double pr = a.z[r] + beta * pOld[r];
    double q = a.A.diag[r] * pr;
    for (int k = 0; k < W; ++k) {
      const int e = b + (k << 5);
      const int c = __ldg(&a.A.col[e]);
      q += a.A.val[e] * (a.z[c] + beta * pOld[c]);
    }
    pNew[r] = pr;
    a.q[r] = q;
    acc[0] += pr * q;
  }
  if (grid_reduce<1>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    a.sc[5] = acc[0];
    a.sc[1] = acc[0] != 0.0 ? a.sc[0] / acc[0] : 0.0;
    a.fl[3] = 0;
  }
}

// x += alpha p ; r -= alpha q ; convergence test on |r|
__global__ void __launch_bounds__(kBlock) k_pcg_xr(PcgArgs a, const double* p) {
  __shared__ double sm[32];
  if (a.fl[0]) return;
  const int n = a.A.n;
  const double al = a.sc[1];
  double acc[1] = {0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    a.x[r] += al * p[r];
    const double rr = a.r[r] - al * a.q[r];
    a.r[r] = rr;
    acc[0] += rr * rr;
  }
  if (grid_reduce<1>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    a.sc[4] = acc[0];
    a.fl[1] += 1;
    if (sqrt(acc[0]) <= a.sc[3]) {
      a.fl[0] = 1;
      a.fl[2] = 1;
    } else if (a.fl[1] >= a.maxit || a.sc[5] == 0.0) {
      a.fl[0] = 1;
      a.fl[2] = 0;
    }
  }
}

// ---------------------------------------------------------------- AMG V-cycle
// Down, part 1: weighted-Jacobi pre-smoothing from zero (x = w D^-1 b) fused with the residual
// r = b - A x (neighbour x computed on the fly); thread per row, SELL-coalesced.  r goes to x2,
// which is free until the up sweep.
__global__ void __launch_bounds__(kBlock) k_amg_resid(const int* done, AmgLevelDev f, double omega) {
  if (*done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < f.n; i += gridDim.x * blockDim.x) {
    const double di = __ldg(&f.diag[i]);
    const double bi = __ldg(&f.b[i]);
    const double xi = __ldg(&f.wdinv[i]) * bi;
    double ax = di * xi;
    const int s = i >> 5;
    const int b = __ldg(&f.sliceOff[s]) + (i & 31);
    const int W = (__ldg(&f.sliceOff[s + 1]) - __ldg(&f.sliceOff[s])) >> 5;
#pragma unroll 4
    for (int k = 0; k < W; ++k) {
      const int e = b + (k << 5);
      const int j = __ldg(&f.col[e]);
      ax += __ldg(&f.val[e]) * (__ldg(&f.wdinv[j]) * __ldg(&f.b[j]));
    }
    f.x[i] = xi;
    f.x2[i] = bi - ax;
  }
}

// Coarse levels (CSR): G consecutive lanes share one row, each lane takes every G-th entry, and
// the partial sums meet through warp shuffles.  Coarse rows are long and there are few of them,
// so splitting rows keeps enough loads in flight.  The warp-level loop bound keeps every lane of
// a warp in the shuffles.
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o, G);
  return v;
}

template <int G>
__global__ void __launch_bounds__(kBlock) k_amg_resid_csr(const int* done, AmgLevelDev f, double omega) {
  if (*done) return;
  const int lane = threadIdx.x & 31, sub = lane % G;
  const int rowsPerWarp = 32 / G;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int base = warp * rowsPerWarp; base < f.n; base += nWarps * rowsPerWarp) {
    const int i = base + lane / G;
    double acc = 0.0;
    if (i < f.n) {
      const int k1 = __ldg(&f.rowOff[i + 1]);
      for (int k = __ldg(&f.rowOff[i]) + sub; k < k1; k += G) {
        const int j = __ldg(&f.col[k]);
        acc += __ldg(&f.val[k]) * (__ldg(&f.wdinv[j]) * __ldg(&f.b[j]));
      }
    }
    acc = group_sum<G>(acc);
    if (i < f.n && sub == 0) {
      const double di = __ldg(&f.diag[i]), bi = __ldg(&f.b[i]);
      const double xi = __ldg(&f.wdinv[i]) * bi;
      f.x[i] = xi;
      f.x2[i] = bi - di * xi - acc;
    }
  }
}

template <int G>
__global__ void __launch_bounds__(kBlock) k_amg_up_csr(const int* done, AmgLevelDev f, const double* e, double omega,
                                                       double corr, double* out) {
  if (*done) return;
  const int lane = threadIdx.x & 31, sub = lane % G;
  const int rowsPerWarp = 32 / G;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int base = warp * rowsPerWarp; base < f.n; base += nWarps * rowsPerWarp) {
    const int i = base + lane / G;
    double acc = 0.0;
    if (i < f.n) {
      const int k1 = __ldg(&f.rowOff[i + 1]);
      for (int k = __ldg(&f.rowOff[i]) + sub; k < k1; k += G) {
        const int j = __ldg(&f.col[k]);
        acc += __ldg(&f.val[k]) * (__ldg(&f.x[j]) + corr * __ldg(&e[__ldg(&f.agg[j])]));
      }
    }
    acc = group_sum<G>(acc);
    if (i < f.n && sub == 0) {
      const double di = __ldg(&f.diag[i]);
      const double xi = __ldg(&f.x[i]) + corr * __ldg(&e[__ldg(&f.agg[i])]);
      out[i] = xi + __ldg(&f.wdinv[i]) * (__ldg(&f.b[i]) - di * xi - acc);
    }
  }
}

// Down, part 2: piecewise-constant restriction b_next[I] = sum of r over the rows of I.
__global__ void __launch_bounds__(kBlock) k_amg_restrict(const int* done, AmgLevelDev f, double* bNext) {
  if (*done) return;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < f.nc; I += gridDim.x * blockDim.x) {
    double acc = 0.0;
    const int m1 = __ldg(&f.memOff[I + 1]);
#pragma unroll 4
    for (int mm = __ldg(&f.memOff[I]); mm < m1; ++mm) acc += f.x2[__ldg(&f.mem[mm])];
    bNext[I] = acc;
  }
}

// Up: prolongate the coarse correction and post-smooth (one weighted-Jacobi sweep) in one pass:
// xt_j = x_j + corr * e[agg(j)] on the fly, out_i = xt_i + w D^-1 (b_i - (A xt)_i).
// On level 0 it also forms r.z for the PCG recurrence.
__global__ void __launch_bounds__(kBlock) k_amg_up(const int* doneFlag, AmgLevelDev f, const double* e, double omega,
                                                   double corr, double* out, int finest, PcgArgs a) {
  __shared__ double sm[32];
  if (*doneFlag) return;
  double acc[1] = {0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < f.n; i += gridDim.x * blockDim.x) {
    const double di = __ldg(&f.diag[i]);
    const double xi = __ldg(&f.x[i]) + corr * __ldg(&e[__ldg(&f.agg[i])]);
    double ax = di * xi;
    const int s = i >> 5;
    const int b = __ldg(&f.sliceOff[s]) + (i & 31);
    const int W = (__ldg(&f.sliceOff[s + 1]) - __ldg(&f.sliceOff[s])) >> 5;
    // unrolled so the col -> agg -> e load chains of several entries are in flight together
#pragma unroll 4
    for (int k = 0; k < W; ++k) {
      const int ee = b + (k << 5);
      const int j = __ldg(&f.col[ee]);
      ax += __ldg(&f.val[ee]) * (__ldg(&f.x[j]) + corr * __ldg(&e[__ldg(&f.agg[j])]));
    }
    const double xn = xi + __ldg(&f.wdinv[i]) * (__ldg(&f.b[i]) - ax);
    out[i] = xn;
    if (finest) acc[0] += f.b[i] * xn;
  }
  if (!finest) return;
  if (grid_reduce<1>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    const double rzOld = a.sc[0];
    a.sc[2] = a.fl[3] ? 0.0 : acc[0] / rzOld;
    a.sc[0] = acc[0];
  }
}

// Coarsest level: x = A^-1 b with the stored dense inverse (one block).  The inverse of the SPD
// coarse matrix is symmetric, so thread i walks column i: consecutive threads read consecutive
// addresses.
__global__ void k_amg_dense_apply(const int* done, int n, const double* inv, const double* b, double* x) {
  if (*done) return;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = w; i < n; i += nw) {  // warp per row, lanes across the row (coalesced)
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += __ldg(&inv[(size_t)i * n + j]) * __ldg(&b[j]);
    s = warp_sum(s);
    if (lane == 0) x[i] = s;
  }
}

// Galerkin values of the next level: one gather list per coarse storage entry.
__global__ void __launch_bounds__(kBlock) k_amg_galerkin(AmgLevelDev f, double* valNext, double* diagNext,
                                                         double* wdinvNext, double omega) {
  const int nT = f.nEntNext + f.nc;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nT; t += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = f.gOff[t]; k < f.gOff[t + 1]; ++k) {
      const int idx = f.gIdx[k];
      s += idx >= 0 ? f.val[idx] : f.diag[-1 - idx];
    }
    if (t < f.nEntNext) {
      valNext[t] = s;
    } else {
      diagNext[t - f.nEntNext] = s;
      wdinvNext[t - f.nEntNext] = omega / s;
    }
  }
}

// Dense inverse of the coarsest matrix by in-place Gauss-Jordan (SPD, no pivoting needed);
// a pivot below 1e-13 of the largest diagonal (singular, all-Neumann systems) gets a zero
// row/column, i.e. the correction ignores the null direction.  One block, shared memory.
__global__ void k_amg_dense_factor(AmgLevelDev c, double* inv) {
  extern __shared__ double A[];
  const int n = c.n;
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) A[t] = 0.0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {  // the coarsest level is always CSR
    A[i * n + i] = c.diag[i];
    for (int k = c.rowOff[i]; k < c.rowOff[i + 1]; ++k) {
      const int j = c.col[k];
      if (j != i) A[i * n + j] += c.val[k];
    }
  }
  __syncthreads();
  __shared__ double dmax;
  if (threadIdx.x == 0) {
    double mx = 0.0;
    for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(A[i * n + i]));
    dmax = mx;
  }
  __syncthreads();
  __shared__ double piv;
  __shared__ int skip;
  for (int k = 0; k < n; ++k) {
    if (threadIdx.x == 0) {
      piv = A[k * n + k];
      skip = fabs(piv) <= 1e-13 * dmax;
    }
    __syncthreads();
    if (skip) {
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        A[k * n + j] = 0.0;
        A[j * n + k] = 0.0;
      }
      __syncthreads();
      continue;
    }
    for (int j = threadIdx.x; j < n; j += blockDim.x)
      if (j != k) A[k * n + j] /= piv;
    __syncthreads();
    if (threadIdx.x == 0) A[k * n + k] = 1.0 / piv;
    __syncthreads();
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
      const int i = t / n, j = t % n;
      if (i == k || j == k) continue;
      A[t] -= A[i * n + k] * A[k * n + j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      if (i != k) A[i * n + k] = -A[i * n + k] * A[k * n + k];
    __syncthreads();
  }
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) inv[t] = A[t];
}

}  // namespace

void bicg_init(const LaunchCfg& lc, const BicgArgs& a) {
  g_launches += 1;
  k_bicg_init<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
}
void bicg_iteration(const LaunchCfg& lc, const BicgArgs& a) {
  {
    ProfScope ps(lc, kKfBicgVector, 0.0);
    k_bicg_p<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
  }
  {
    ProfScope ps(lc, kKfBicgSpmv, lc.ab ? lc.ab->bicg_spmv(a.nc) : 0.0);
    k_bicg_v<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
  }
  {
    ProfScope ps(lc, kKfBicgVector, 0.0);
    k_bicg_s<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
  }
  {
    ProfScope ps(lc, kKfBicgSpmv, lc.ab ? lc.ab->bicg_spmv(a.nc) : 0.0);
    k_bicg_t<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
  }
  {
    ProfScope ps(lc, kKfBicgVector, 0.0);
    k_bicg_x<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
  }
}

void pcg_init(const LaunchCfg& lc, const PcgArgs& a) {
  g_launches += 1;
  k_pcg_init<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
}

static int blocks_for(int n, int cap) { return std::max(1, std::min(cap, (n + kBlock - 1) / kBlock)); }

constexpr int kCoarseLanes = 8;  // lanes per row on the CSR coarse levels

static void vcycle(const LaunchCfg& lc, const PcgArgs& a, const AmgDev* amg) {
  const int L = amg->nLevels;
  // level 0 right-hand side is the PCG residual
  {
    const AmgLevelDev& f = amg->lv[0];
    ProfScope ps(lc, kKfAmgResid0, 0.0, 2);
    k_amg_resid<<<blocks_for(f.n, lc.rowBlocks), kBlock, 0, lc.stream>>>(a.fl, f, amg->omega);
    k_amg_restrict<<<blocks_for(f.nc, lc.rowBlocks), kBlock, 0, lc.stream>>>(a.fl, f, amg->lv[1].b);
  }
  {
    ProfScope ps(lc, kKfAmgCoarse, 0.0, 3 * L - 6);
    for (int l = 1; l + 1 < L; ++l) {
      const AmgLevelDev& f = amg->lv[l];
      k_amg_resid_csr<kCoarseLanes><<<blocks_for(f.n * kCoarseLanes, lc.rowBlocks), kBlock, 0, lc.stream>>>(
          a.fl, f, amg->omega);
      k_amg_restrict<<<blocks_for(f.nc, lc.rowBlocks), kBlock, 0, lc.stream>>>(a.fl, f, amg->lv[l + 1].b);
    }
    const AmgLevelDev& c = amg->lv[L - 1];
    k_amg_dense_apply<<<1, 1024, 0, lc.stream>>>(a.fl, c.n, amg->dense, c.b, c.x);
    for (int l = L - 2; l >= 1; --l) {
      const AmgLevelDev& f = amg->lv[l];
      // correction from the coarser level: its smoothed solution (x2), or x on the coarsest
      const double* e = (l + 1 == L - 1) ? amg->lv[l + 1].x : amg->lv[l + 1].x2;
      k_amg_up_csr<kCoarseLanes><<<blocks_for(f.n * kCoarseLanes, lc.rowBlocks), kBlock, 0, lc.stream>>>(
          a.fl, f, e, amg->omega, amg->corr, f.x2);
    }
  }
  {
    const AmgLevelDev& f = amg->lv[0];
    const double* e = (L == 2) ? amg->lv[1].x : amg->lv[1].x2;
    ProfScope ps(lc, kKfAmgUp0, 0.0);
    k_amg_up<<<blocks_for(f.n, lc.rowBlocks), kBlock, 0, lc.stream>>>(a.fl, f, e, amg->omega, amg->corr, a.z, 1, a);
  }
}

void pcg_precondition(const LaunchCfg& lc, const PcgArgs& a, const AmgDev* amg) {
  if (!amg || amg->nLevels < 2) {
    g_launches += 1;
    k_pcg_jacobi<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
  } else if (amg->graph) {
    g_launches += amg->graphKernels;
    cudaGraphLaunch(amg->graph, lc.stream);
  } else {
    vcycle(lc, a, amg);
  }
}

// Records one V-cycle into a CUDA graph.  Every pointer and scalar the V-cycle kernels read is
// fixed for the life of the hierarchy (values change on refresh, addresses do not), so the
// graph is captured once and replayed for every preconditioner application.
cudaError_t amg_capture_graph(const LaunchCfg& lc, const PcgArgs& a, AmgDev& amg) {
  if (amg.graph) {
    cudaGraphExecDestroy(amg.graph);
    amg.graph = nullptr;
  }
  LaunchCfg quiet = lc;
  quiet.prof = nullptr;
  const long long before = g_launches.load();
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(lc.stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  vcycle(quiet, a, &amg);
  e = cudaStreamEndCapture(lc.stream, &g);
  amg.graphKernels = (int)(g_launches.load() - before);
  g_launches -= amg.graphKernels;
  if (e != cudaSuccess) return e;
  e = cudaGraphInstantiate(&amg.graph, g, 0);
  cudaGraphDestroy(g);
  return e;
}

void pcg_iteration(const LaunchCfg& lc, const PcgArgs& a, int it, const AmgDev* amg) {
  const double* pOld = (it & 1) ? a.p1 : a.p0;
  double* pNew = (it & 1) ? a.p0 : a.p1;
  {
    ProfScope ps(lc, kKfPcgSpmv, lc.ab ? lc.ab->pcg_spmv() : 0.0);
    k_pcg_pq<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a, pOld, pNew);
  }
  {
    ProfScope ps(lc, kKfPcgUpdate, 0.0);
    k_pcg_xr<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a, pNew);
  }
  pcg_precondition(lc, a, amg);
}

void amg_refresh(const LaunchCfg& lc, AmgDev& amg) {
  for (int l = 0; l + 1 < amg.nLevels; ++l) {
    AmgLevelDev& f = amg.lv[l];
    AmgLevelDev& c = amg.lv[l + 1];
    g_launches += 1;
    k_amg_galerkin<<<blocks_for(f.nEntNext + f.nc, lc.rowBlocks), kBlock, 0, lc.stream>>>(f, c.val, c.diag,
                                                                                          c.wdinv, amg.omega);
  }
  const AmgLevelDev& c = amg.lv[amg.nLevels - 1];
  const size_t smem = sizeof(double) * (size_t)c.n * c.n;
  cudaFuncSetAttribute(k_amg_dense_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  g_launches += 1;
  k_amg_dense_factor<<<1, 1024, smem, lc.stream>>>(c, amg.dense);
}

}  // namespace anb
