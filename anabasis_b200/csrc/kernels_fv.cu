// Finite-volume face/cell kernels of the SIMPLE outer iteration (sm_100a).
//
// Every kernel is cell-centric over the SELL-32 layout: thread r owns row r, walks its
// off-diagonal slots (one per neighbour, each slot naming the connecting face) and its boundary
// faces, and accumulates diagonal, right-hand side and divergence in registers.  Each row writes
// only its own outputs, so the reference's FP64 atomicAdd scatters (main.cu:56-58) become
// deterministic gathers; a face's flux is written by its owner row.
#include <cstdlib>
#include <mutex>
#include <string>
#include <unordered_map>

#include "kernels.cuh"

namespace anb {

namespace {

// Slot indices of row r in registers for a compile-time bound WM on the slice width (slots past
// the row's width read as face -1, column r), so every load of the slot loop below can be issued
// before the first result is needed.  Returns the row's first storage index.
template <int WM>
__device__ __forceinline__ int slot_regs(const DMesh& m, int r, int (&f)[WM], int (&c)[WM]) {
  const int s = r >> 5;
  const int b0 = __ldg(&m.sliceOff[s]);
  const int W = (__ldg(&m.sliceOff[s + 1]) - b0) >> 5;
  const int base = b0 + (r & 31);
#pragma unroll
  for (int k = 0; k < WM; ++k) {
    f[k] = -1;
    c[k] = r;
    if (k < W) {
      f[k] = __ldg(&m.slotFace[base + (k << 5)]);
      c[k] = __ldg(&m.col[base + (k << 5)]);
    }
  }
  return base;
}

// ---- least-squares gradient: main.cu:1403-1440 on the moments of main.cu:1159-1251 ----------
template <int NF>
__device__ __forceinline__ void grad_slot(const DMesh& m, const GradArgs& a, int c, const double (&ccr)[3],
                                          const double (&pr)[NF], double (&b)[NF][3]) {
  // r = cc_c - cc_r from the cell centres (neighbour centres are L2-resident gathers): for the
  // owner row this is the face's d = cc_N - cc_P, for the neighbour row its negation, bit for bit
  const double r0 = __ldg(&m.cc[3 * c]) - ccr[0], r1 = __ldg(&m.cc[3 * c + 1]) - ccr[1],
               r2 = __ldg(&m.cc[3 * c + 2]) - ccr[2];
  const double w = 1.0 / fmax(r0 * r0 + r1 * r1 + r2 * r2, 1e-30);
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    const double dp = w * (__ldg(&a.phi[f][c]) - pr[f]);
    b[f][0] += r0 * dp;
    b[f][1] += r1 * dp;
    b[f][2] += r2 * dp;
  }
}

template <int NF, int WM>
__global__ void __launch_bounds__(kBlock) k_lsq_grad(DMesh m, GradArgs a) {
  const int C = m.nCells;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double pr[NF], b[NF][3];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      pr[f] = __ldg(&a.phi[f][r]);
      b[f][0] = b[f][1] = b[f][2] = 0.0;
    }
    const double ccr[3] = {__ldg(&m.cc[3 * r]), __ldg(&m.cc[3 * r + 1]), __ldg(&m.cc[3 * r + 2])};
    if constexpr (WM > 0) {
      int fs[WM], cs[WM];
      slot_regs<WM>(m, r, fs, cs);
#pragma unroll
      for (int k = 0; k < WM; ++k)
        if (fs[k] >= 0) grad_slot<NF>(m, a, cs[k], ccr, pr, b);
    } else {
      int W;
      const int base = row_base(m, r, W);
      for (int k = 0; k < W; ++k) {
        const int e = base + (k << 5);
        if (__ldg(&m.slotFace[e]) < 0) break;
        grad_slot<NF>(m, a, __ldg(&m.col[e]), ccr, pr, b);
      }
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      const unsigned ty = __ldg(&m.bType[bf]);
      const double* dd = m.bnd[bf].d;
      const double r0 = dd[0], r1 = dd[1], r2 = dd[2];
      const double w = 1.0 / fmax(r0 * r0 + r1 * r1 + r2 * r2, 1e-30);
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        if (!(ty & a.bit[f])) continue;  // Neumann: phi_f = phi_P contributes nothing
        const double dp = w * (a.bval[f][bf] - pr[f]);
        b[f][0] += r0 * dp;
        b[f][1] += r1 * dp;
        b[f][2] += r2 * dp;
      }
    }
    const double* M = m.minv + 6 * r;
    const double m0 = M[0], m1 = M[1], m2 = M[2], m3 = M[3], m4 = M[4], m5 = M[5];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      double* g = a.g[f];
      g[r] = m0 * b[f][0] + m1 * b[f][1] + m2 * b[f][2];
      g[C + r] = m1 * b[f][0] + m3 * b[f][1] + m4 * b[f][2];
      g[2 * C + r] = m2 * b[f][0] + m4 * b[f][1] + m5 * b[f][2];
    }
  }
}

// ---- momentum: K25,K4,K2,K3,K5,K6 + rhs-only K26,K9,K7,K8,K10 for V and W in one pass ------
// main.cu:1678-1896 (assembly), 1686-1695 (relaxation), 1787-1802 (rAU), loop 3350-3405.
// Contributions of internal slot e (neighbour c) of row r: the off-diagonal value, and the
// diagonal and right-hand-side increments of the row.  Row values (U, the 9 velocity-gradient
// components) come in registers; owner-orientation P/N values are selected, not re-loaded, so
// the arithmetic is that of a face visited from either side.
template <class M>
__device__ __forceinline__ void momentum_slot(const DMesh& m, const MomArgsT<M>& a, int C, int r, int e, int c,
                                              const double (&ur)[3], const double (&gr)[9], double& val,
                                              double& dDiag, double (&dRhs)[3]) {
  const bool own = r < c;
  double lam, g, t[3], d[3];
  load_slot(m, e, lam, g, t, d);
  const double l1 = 1.0 - lam;
  const double alpha = a.mu * g;
  const double S0 = t[0] + g * d[0], S1 = t[1] + g * d[1], S2 = t[2] + g * d[2];
  double uc[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double x = __ldg(&a.U[q * C + c]);
    uc[q] = l1 * (own ? ur[q] : x) + lam * (own ? x : ur[q]);
  }
  const double F = a.rho * (uc[0] * S0 + uc[1] * S1 + uc[2] * S2);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double gq[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double x = __ldg(&a.G[(3 * q + k) * C + c]);
      gq[k] = l1 * (own ? gr[3 * q + k] : x) + lam * (own ? x : gr[3 * q + k]);
    }
    dRhs[q] = a.mu * (gq[0] * t[0] + gq[1] * t[1] + gq[2] * t[2]);
  }
  if (own) {
    val = -alpha + F * lam;
    dDiag = alpha + F * l1;
  } else {
    val = -alpha - F * l1;
    dDiag = alpha - F * lam;
  }
}

template <class M, int WM>
__global__ void __launch_bounds__(kBlock, 3) k_momentum(DMesh m, MomArgsT<M> a) {
  const int C = m.nCells;
  const bool full = !a.rhsOnly;
  const double* G = a.G;
  const double rho = a.rho, mu = a.mu;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    const double V = m.vol[r];
    double rhs0 = -G[9 * C + r] * V, rhs1 = -G[10 * C + r] * V, rhs2 = -G[11 * C + r] * V;
    double diag = 0.0;
    const double ur[3] = {__ldg(&a.U[r]), __ldg(&a.U[C + r]), __ldg(&a.U[2 * C + r])};
    double gr[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) gr[k] = __ldg(&G[k * C + r]);
    auto add = [&](int e, int c, double& val) {
      double dd, dr[3];
      momentum_slot(m, a, C, r, e, c, ur, gr, val, dd, dr);
      diag += dd;
      if (r < c) {
        rhs0 += dr[0]; rhs1 += dr[1]; rhs2 += dr[2];
      } else {
        rhs0 -= dr[0]; rhs1 -= dr[1]; rhs2 -= dr[2];
      }
    };
    if constexpr (WM > 0) {
      // every load of the row first, the matrix stores after the loop
      int fs[WM], cs[WM];
      const int base = slot_regs<WM>(m, r, fs, cs);
      double vals[WM];
#pragma unroll
      for (int k = 0; k < WM; ++k) {
        vals[k] = 0.0;
        if (fs[k] < 0 || !(__ldg(&m.slotFlags[base + (k << 5)]) & 1)) continue;
        add(base + (k << 5), cs[k], vals[k]);
      }
      if (full) {
        const int W = (__ldg(&m.sliceOff[(r >> 5) + 1]) - __ldg(&m.sliceOff[r >> 5])) >> 5;
#pragma unroll
        for (int k = 0; k < WM; ++k)
          if (k < W) a.val[base + (k << 5)] = (M)vals[k];
      }
    } else {
      int W;
      const int base = row_base(m, r, W);
      for (int k = 0; k < W; ++k) {
        const int e = base + (k << 5);
        const int f = __ldg(&m.slotFace[e]);
        double v = 0.0;
        if (f >= 0 && (__ldg(&m.slotFlags[e]) & 1)) add(e, __ldg(&m.col[e]), v);
        if (full) a.val[e] = (M)v;
      }
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      if (!(__ldg(&m.bFlags[bf]) & 1)) continue;
      double g, t[3], S[3], d[3];
      load_bnd(m.bnd, bf, g, t, S, d);
      const unsigned ty = __ldg(&m.bType[bf]);
      const double alpha = mu * g;
      const double bu = m.bVal[bf], bv = m.bVal[m.nBoundary + bf], bw = m.bVal[2 * m.nBoundary + bf];
      const double ub = (ty & 1u) ? bu : ur[0], vb = (ty & 2u) ? bv : ur[1], wb = (ty & 4u) ? bw : ur[2];
      const double F = rho * (ub * S[0] + vb * S[1] + wb * S[2]);
      diag += (ty & 1u) ? alpha : F;  // the matrix carries the u-component BC types
      if (ty & 1u) rhs0 += alpha * bu + mu * (gr[0] * t[0] + gr[1] * t[1] + gr[2] * t[2]) - F * bu;
      if (ty & 2u) rhs1 += alpha * bv + mu * (gr[3] * t[0] + gr[4] * t[1] + gr[5] * t[2]) - F * bv;
      if (ty & 4u) rhs2 += alpha * bw + mu * (gr[6] * t[0] + gr[7] * t[1] + gr[8] * t[2]) - F * bw;
    }
    const double q0 = a.Q[r], q1 = a.Q[C + r], q2 = a.Q[2 * C + r];
    if (full) {
      if (a.relax) {
        const double invR = 1.0 / a.uRelax;
        const double aP = diag;
        diag = aP * invR;
        rhs0 += (invR - 1.0) * aP * q0;                 // K5 on the u pass
        const double aPold = diag * a.uRelax;          // K10 on the v and w passes
        rhs1 += (invR - 1.0) * aPold * q1;
        rhs2 += (invR - 1.0) * aPold * q2;
      }
      a.diag[r] = (M)diag;
      a.rau[r] = fabs(diag) > 1e-30 ? V / diag : 0.0;
    } else if (a.relax) {                                 // K10 for every re-solve
      const double invR = 1.0 / a.uRelax;
      const double aPold = (double)a.diag[r] * a.uRelax;
      rhs0 += (invR - 1.0) * aPold * q0;
      rhs1 += (invR - 1.0) * aPold * q1;
      rhs2 += (invR - 1.0) * aPold * q2;
    }
    a.rhs[r] = rhs0;
    a.rhs[C + r] = rhs1;
    a.rhs[2 * C + r] = rhs2;
  }
}

// ---- pressure matrix (K11,K12) + Rhie-Chow flux (K14) + continuity (K15) ------------------
// main.cu:1898-1950, 1474-1536, launch sequence 3407-3452.  The plain slot loop measured faster
// here than the register-staged form of the other face kernels (many gathers per slot).
template <class M>
__global__ void __launch_bounds__(kBlock) k_pressure_rc(DMesh m, PresArgsT<M> a) {
  const int C = m.nCells, nI = m.nInternal;
  const double* U0 = a.Us;
  const double* U1 = a.Us + C;
  const double* U2 = a.Us + 2 * C;
  const double* Gp = a.Gp;
  const double rho = a.rho;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double pd = 0.0, div = 0.0;
    const double rAUr = a.rau[r];
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) {
        a.val[e] = M(0);
        continue;
      }
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      double lam, g, t[3], d[3];
      load_slot(m, e, lam, g, t, d);
      const int P = own ? r : c, N = own ? c : r;
      const double l1 = 1.0 - lam;
      const double rAUf = l1 * a.rau[P] + lam * a.rau[N];
      if (__ldg(&m.slotFlags[e]) & 1) {
        const double coeff = g * rAUf;
        a.val[e] = (M)(-coeff);
        pd += coeff;
      } else {
        a.val[e] = M(0);
      }
      const double S0 = t[0] + g * d[0], S1 = t[1] + g * d[1], S2 = t[2] + g * d[2];
      const double ub = l1 * U0[P] + lam * U0[N], vb = l1 * U1[P] + lam * U1[N], wb = l1 * U2[P] + lam * U2[N];
      const double gx = l1 * Gp[P] + lam * Gp[N], gy = l1 * Gp[C + P] + lam * Gp[C + N],
                   gz = l1 * Gp[2 * C + P] + lam * Gp[2 * C + N];
      const double phiI = rho * (ub * S0 + vb * S1 + wb * S2);
      const double rc = rho * g * rAUf * ((a.P[N] - a.P[P]) - (gx * d[0] + gy * d[1] + gz * d[2]));
      const double phi = phiI - rc;
      if (own) {
        div += phi;
        a.phiStar[f] = phi;
      } else {
        div -= phi;
      }
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      double g, t[3], S[3], d[3];
      load_bnd(m.bnd, bf, g, t, S, d);
      const unsigned ty = __ldg(&m.bType[bf]);
      if ((ty & 8u) && (__ldg(&m.bFlags[bf]) & 1)) pd += g * rAUr;
      const double uf = (ty & 1u) ? m.bVal[bf] : U0[r];
      const double vf = (ty & 2u) ? m.bVal[m.nBoundary + bf] : U1[r];
      const double wf = (ty & 4u) ? m.bVal[2 * m.nBoundary + bf] : U2[r];
      const double phi = rho * (uf * S[0] + vf * S[1] + wf * S[2]);
      div += phi;
      a.phiStar[nI + bf] = phi;
    }
    a.diag[r] = (M)pd;
    if (a.wdinv) a.wdinv[r] = (M)(a.omega / pd);  // level-0 smoother weight, always from the current matrix
    a.divStar[r] = div;
    a.b[r] = -div;
    a.pc[r] = 0.0;
  }
}

// ---- non-orthogonal divergence (K16) + pressure rhs (K17): main.cu:1538-1604 --------------
__device__ __forceinline__ double nonorth_slot(const DMesh& m, const NonOrthArgs& a, int C, int r, int e, int c,
                                               double rAUr, const double (&gr)[3]) {
  const bool own = r < c;
  double lam, g, t[3], d[3];
  load_slot(m, e, lam, g, t, d);
  const double l1 = 1.0 - lam;
  const double rc_ = __ldg(&a.rau[c]);
  const double rAUf = l1 * (own ? rAUr : rc_) + lam * (own ? rc_ : rAUr);
  double gf[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double y = __ldg(&a.Gc[q * C + c]);
    gf[q] = l1 * (own ? gr[q] : y) + lam * (own ? y : gr[q]);
  }
  const double flux = rAUf * (gf[0] * t[0] + gf[1] * t[1] + gf[2] * t[2]);
  return own ? flux : -flux;
}

template <int WM>
__global__ void __launch_bounds__(kBlock, 6) k_nonorth_rhs(DMesh m, NonOrthArgs a) {
  const int C = m.nCells;
  const double* Gc = a.Gc;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double dno = 0.0;
    const double rAUr = __ldg(&a.rau[r]);
    const double gr[3] = {__ldg(&Gc[r]), __ldg(&Gc[C + r]), __ldg(&Gc[2 * C + r])};
    if constexpr (WM > 0) {
      int fs[WM], cs[WM];
      const int base = slot_regs<WM>(m, r, fs, cs);
#pragma unroll
      for (int k = 0; k < WM; ++k)
        if (fs[k] >= 0 && (__ldg(&m.slotFlags[base + (k << 5)]) & 2))
          dno += nonorth_slot(m, a, C, r, base + (k << 5), cs[k], rAUr, gr);
    } else {
      int W;
      const int base = row_base(m, r, W);
      for (int k = 0; k < W; ++k) {
        const int e = base + (k << 5);
        const int f = __ldg(&m.slotFace[e]);
        if (f < 0) break;
        if (!(__ldg(&m.slotFlags[e]) & 2)) continue;
        dno += nonorth_slot(m, a, C, r, e, __ldg(&m.col[e]), rAUr, gr);
      }
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      if (!(__ldg(&m.bType[bf]) & 8u) || !(__ldg(&m.bFlags[bf]) & 2)) continue;
      const double* t = m.bnd[bf].t;
      dno += rAUr * (gr[0] * t[0] + gr[1] * t[1] + gr[2] * t[2]);
    }
    a.b[r] = -a.divBase[r] + dno;
  }
}

// ---- flux correction (K16 + K19) + continuity (K15) [+ K21, K20, step statistics] ----------
// main.cu:1615-1658, 1523-1536, 3568-3603.
// Corrected flux of internal slot e (face f, neighbour c) of row r, in the face's owner
// orientation: both rows of a face evaluate the same expression on the same values, so the
// owner's phi and the neighbour's are equal bit for bit.  Row values (rAU, p', grad p') come in
// registers; all loads are read-only.
__device__ __forceinline__ double flux_slot(const DMesh& m, const FluxArgs& a, int C, int r, int e, int f, int c,
                                            double rAUr, double pcr, const double (&gr)[3], bool& own) {
  own = r < c;
  double lam, g, t[3], d[3];
  load_slot(m, e, lam, g, t, d);
  const double rAUc = __ldg(&a.rau[c]), pcc = __ldg(&a.pc[c]);
  const double rP = own ? rAUr : rAUc, rN = own ? rAUc : rAUr;
  const double pP = own ? pcr : pcc, pN = own ? pcc : pcr;
  const double l1 = 1.0 - lam;
  const double rAUf = l1 * rP + lam * rN;
  double phiNO = 0.0;
  if (__ldg(&m.slotFlags[e]) & 2) {
    const double c0 = __ldg(&a.Gc[c]), c1 = __ldg(&a.Gc[C + c]), c2 = __ldg(&a.Gc[2 * C + c]);
    const double gx = l1 * (own ? gr[0] : c0) + lam * (own ? c0 : gr[0]);
    const double gy = l1 * (own ? gr[1] : c1) + lam * (own ? c1 : gr[1]);
    const double gz = l1 * (own ? gr[2] : c2) + lam * (own ? c2 : gr[2]);
    phiNO = rAUf * (gx * t[0] + gy * t[1] + gz * t[2]);
  }
  return __ldg(&a.phiStar[f]) - g * rAUf * (pN - pP) - phiNO;
}

template <int WM>
__global__ void __launch_bounds__(kBlock) k_flux_final(DMesh m, FluxArgs a) {
  __shared__ double sm[9 * 32];
  const int C = m.nCells, nI = m.nInternal;
  const double* Gc = a.Gc;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double div = 0.0;
    const double pcr = __ldg(&a.pc[r]), rAUr = __ldg(&a.rau[r]);
    const double gr[3] = {__ldg(&Gc[r]), __ldg(&Gc[C + r]), __ldg(&Gc[2 * C + r])};
    if constexpr (WM > 0) {
      // every load of the row first, the owner's flux stores after the loop
      int fs[WM], cs[WM];
      const int base = slot_regs<WM>(m, r, fs, cs);
      double ph[WM];
#pragma unroll
      for (int k = 0; k < WM; ++k) {
        ph[k] = 0.0;
        if (fs[k] < 0) continue;
        bool own;
        ph[k] = flux_slot(m, a, C, r, base + (k << 5), fs[k], cs[k], rAUr, pcr, gr, own);
        if (own) {
          div += ph[k];
        } else {
          div -= ph[k];
          fs[k] = -1;
        }
      }
#pragma unroll
      for (int k = 0; k < WM; ++k)
        if (fs[k] >= 0) a.phi[fs[k]] = ph[k];
    } else {
      int W;
      const int base = row_base(m, r, W);
      for (int k = 0; k < W; ++k) {
        const int e = base + (k << 5);
        const int f = __ldg(&m.slotFace[e]);
        if (f < 0) break;
        bool own;
        const double phi = flux_slot(m, a, C, r, e, f, __ldg(&m.col[e]), rAUr, pcr, gr, own);
        if (own) {
          div += phi;
          a.phi[f] = phi;
        } else {
          div -= phi;
        }
      }
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      const unsigned ty = __ldg(&m.bType[bf]);
      double phi = a.phiStar[nI + bf];
      if ((ty & 8u) && (__ldg(&m.bFlags[bf]) & 2)) {
        const double g = m.bnd[bf].g;
        const double* t = m.bnd[bf].t;
        const double phiNO = rAUr * (gr[0] * t[0] + gr[1] * t[1] + gr[2] * t[2]);
        phi = phi - g * rAUr * (m.bVal[3 * m.nBoundary + bf] - pcr) - phiNO;
      }
      div += phi;
      a.phi[nI + bf] = phi;
    }
    a.divCorr[r] = div;
    if (a.update) {
      const double pOld = a.P[r];
      const double pNew = pOld + a.pRelax * pcr;
      a.P[r] = pNew;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const double uo = a.U[q * C + r];
        const double un = a.Us[q * C + r] - rAUr * gr[q];
        a.U[q * C + r] = un;
        const double dd = un - uo;
        acc[2 * q] += dd * dd;
        acc[2 * q + 1] += un * un;
      }
      const double dp = pNew - pOld;
      acc[6] += dp * dp;
      acc[7] += pNew * pNew;
      // a non-finite divergence must reach the host's divergence test: fmax would drop a NaN
      const double ad = fabs(div);
      acc[8] = (ad == ad) ? fmax(acc[8], ad) : INFINITY;
    }
  }
  if (!a.update) return;
  if (grid_reduce<9>(acc, 1u << 8, a.red, sm) && threadIdx.x == 0)
    for (int q = 0; q < 9; ++q) a.stats[q] = acc[q];
}

// ---- flux correction, face-parallel form -------------------------------------------------
// Each internal face's corrected flux once, in its owner orientation, by one thread (the
// expression of flux_slot for the owner row), then a row kernel that sums the divergence in slot
// order from the stored fluxes and applies the updates of k_flux_final.
__global__ void __launch_bounds__(kBlock) k_flux_faces(DMesh m, FluxArgs a) {
  const int C = m.nCells;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < m.nInternal; f += gridDim.x * blockDim.x) {
    const int P = __ldg(&m.fOwner[f]), N = __ldg(&m.fNeigh[f]);
    double lam, g, t[3], d[3];
    load_face(m.face, f, lam, g, t, d);
    const double rP = __ldg(&a.rau[P]), rN = __ldg(&a.rau[N]);
    const double pP = __ldg(&a.pc[P]), pN = __ldg(&a.pc[N]);
    const double l1 = 1.0 - lam;
    const double rAUf = l1 * rP + lam * rN;
    double phiNO = 0.0;
    if (__ldg(&m.fFlags[f]) & 2) {
      const double gx = l1 * __ldg(&a.Gc[P]) + lam * __ldg(&a.Gc[N]);
      const double gy = l1 * __ldg(&a.Gc[C + P]) + lam * __ldg(&a.Gc[C + N]);
      const double gz = l1 * __ldg(&a.Gc[2 * C + P]) + lam * __ldg(&a.Gc[2 * C + N]);
      phiNO = rAUf * (gx * t[0] + gy * t[1] + gz * t[2]);
    }
    a.phi[f] = __ldg(&a.phiStar[f]) - g * rAUf * (pN - pP) - phiNO;
  }
}

template <int WM>
__global__ void __launch_bounds__(kBlock) k_flux_cells(DMesh m, FluxArgs a) {
  __shared__ double sm[9 * 32];
  const int C = m.nCells, nI = m.nInternal;
  const double* Gc = a.Gc;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double div = 0.0;
    const double pcr = __ldg(&a.pc[r]), rAUr = __ldg(&a.rau[r]);
    const double gr[3] = {__ldg(&Gc[r]), __ldg(&Gc[C + r]), __ldg(&Gc[2 * C + r])};
    if constexpr (WM > 0) {
      int fs[WM], cs[WM];
      slot_regs<WM>(m, r, fs, cs);
#pragma unroll
      for (int k = 0; k < WM; ++k) {
        if (fs[k] < 0) continue;
        const double ph = a.phi[fs[k]];
        div += r < cs[k] ? ph : -ph;
      }
    } else {
      int W;
      const int base = row_base(m, r, W);
      for (int k = 0; k < W; ++k) {
        const int e = base + (k << 5);
        const int f = __ldg(&m.slotFace[e]);
        if (f < 0) break;
        const double ph = a.phi[f];
        div += r < __ldg(&m.col[e]) ? ph : -ph;
      }
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      const unsigned ty = __ldg(&m.bType[bf]);
      double phi = a.phiStar[nI + bf];
      if ((ty & 8u) && (__ldg(&m.bFlags[bf]) & 2)) {
        const double g = m.bnd[bf].g;
        const double* t = m.bnd[bf].t;
        const double phiNO = rAUr * (gr[0] * t[0] + gr[1] * t[1] + gr[2] * t[2]);
        phi = phi - g * rAUr * (m.bVal[3 * m.nBoundary + bf] - pcr) - phiNO;
      }
      div += phi;
      a.phi[nI + bf] = phi;
    }
    a.divCorr[r] = div;
    if (a.update) {
      const double pOld = a.P[r];
      const double pNew = pOld + a.pRelax * pcr;
      a.P[r] = pNew;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const double uo = a.U[q * C + r];
        const double un = a.Us[q * C + r] - rAUr * gr[q];
        a.U[q * C + r] = un;
        const double dd = un - uo;
        acc[2 * q] += dd * dd;
        acc[2 * q + 1] += un * un;
      }
      const double dp = pNew - pOld;
      acc[6] += dp * dp;
      acc[7] += pNew * pNew;
      const double ad = fabs(div);
      acc[8] = (ad == ad) ? fmax(acc[8], ad) : INFINITY;
    }
  }
  if (!a.update) return;
  if (grid_reduce<9>(acc, 1u << 8, a.red, sm) && threadIdx.x == 0)
    for (int q = 0; q < 9; ++q) a.stats[q] = acc[q];
}

// ---- patch force: main.cu:2828-2933 (single block, deterministic order) -------------------
__global__ void k_patch_force(DMesh m, int b0, int b1, int sign, double mu, const double* bA, const double* bN,
                              const double* U, const double* P, double* out) {
  __shared__ double sm[16 * 32];
  const int C = m.nCells;
  double v[16];
  for (int q = 0; q < 16; ++q) v[q] = 0.0;
  v[11] = -1.0e308;  // -min dn (as max)
  v[12] = -1.0e308;  // max dn
  v[13] = -1.0e308;  // max |Ut|
  v[14] = -1.0e308;  // max shear
  for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x) {
    const int r = m.bOwner[b];
    const double A = bA[b];
    if (A <= 1.0e-300) continue;
    double n0 = (double)sign * bN[3 * b], n1 = (double)sign * bN[3 * b + 1], n2 = (double)sign * bN[3 * b + 2];
    const double nm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    if (nm <= 1.0e-300) continue;
    const double inv = 1.0 / nm;
    n0 *= inv; n1 *= inv; n2 *= inv;
    const double* d = m.bnd[b].d;  // x_f - cc_P
    const double dx0 = -d[0], dx1 = -d[1], dx2 = -d[2];
    double dn = dx0 * n0 + dx1 * n1 + dx2 * n2;
    if (dn <= 1.0e-14) dn = fabs(dn);
    if (dn <= 1.0e-14) dn = sqrt(dx0 * dx0 + dx1 * dx1 + dx2 * dx2);
    if (dn <= 1.0e-14) continue;
    const double u0 = U[r], u1 = U[C + r], u2 = U[2 * C + r];
    const double Un = u0 * n0 + u1 * n1 + u2 * n2;
    const double t0 = u0 - Un * n0, t1 = u1 - Un * n1, t2 = u2 - Un * n2;
    const double Ut = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
    const double pr = P[r];
    const double nn[3] = {n0, n1, n2}, tt[3] = {t0, t1, t2};
#pragma unroll
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
  }
  block_reduce<16>(v, (1u << 11) | (1u << 12) | (1u << 13) | (1u << 14), sm);
  if (threadIdx.x == 0) {
    for (int q = 0; q < 11; ++q) out[q] = v[q];
    out[11] = v[10] > 0 ? -v[11] : 0.0;
    out[12] = v[10] > 0 ? v[12] : 0.0;
    out[13] = v[10] > 0 ? v[13] : 0.0;
    out[14] = v[10] > 0 ? v[14] : 0.0;
  }
}

// ---- extra pressure passes (nPressureCorr, main.cu:3521-3567) ------------------------------
// b = -divCorr (kernel_build_pressure_rhs_minus_div, main.cu:1606-1613; the reference's pressure
// anchor is off, main.cu:3294) and dp' = 0 for the pass's solve from zero.
__global__ void __launch_bounds__(kBlock) k_pass_rhs(int n, const double* divCorr, double* b, double* dx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    b[i] = -divCorr[i];
    dx[i] = 0.0;
  }
}

// y += s x (kernel_add_scaled_inplace, main.cu:1442-1445)
__global__ void __launch_bounds__(kBlock) k_add_scaled(int n, double s, const double* x, double* y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += s * x[i];
}

// Cell-field permutation for the host/device boundary (input <-> layout numbering).  The index is
// read once per row and every component's gather issued before its store.
__global__ void __launch_bounds__(kBlock) k_permute_cells(PermuteArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const int j = a.idx[i];
    double v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (q < a.comps) v[q] = a.src[q][j];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (q < a.comps) a.dst[q][i] = v[q];
  }
}

// Relative change of the three momentum iterates (main.cu:3377-3379): per component the sum of
// (after - before)^2 and of after^2, combined in block order into out[0..5].
__global__ void __launch_bounds__(kBlock) k_relchg3(int n, const double* before, const double* after, Reducer red,
                                                    double* out) {
  __shared__ double sm[6 * 32];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double a = after[(size_t)q * n + i];
      const double d = a - before[(size_t)q * n + i];
      acc[2 * q] += d * d;
      acc[2 * q + 1] += a * a;
    }
  }
  if (grid_reduce<6>(acc, 0u, red, sm) && threadIdx.x == 0)
    for (int q = 0; q < 6; ++q) out[q] = acc[q];
}

}  // namespace

void launch_pass_rhs(const LaunchCfg& lc, int n, const double* divCorr, double* b, double* dx) {
  g_launches += 1;
  k_pass_rhs<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(n, divCorr, b, dx);
}
void launch_permute_cells(const LaunchCfg& lc, const PermuteArgs& a) {
  g_launches += 1;
  k_permute_cells<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(a);
}
void launch_add_scaled(const LaunchCfg& lc, int n, double s, const double* x, double* y) {
  g_launches += 1;
  k_add_scaled<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(n, s, x, y);
}
void launch_relchg3(const LaunchCfg& lc, int n, const double* before, const double* after, Reducer red,
                    double* out) {
  g_launches += 1;
  k_relchg3<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(n, before, after, red, out);
}

std::atomic<long long> g_launches{0};

int resident_blocks(const void* kernel) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kBlock, 0) != cudaSuccess) {
    cudaGetLastError();
    n = 0;  // unknown: the caller keeps its cap
  }
  cache.emplace(kernel, n);
  return n;
}

// Compulsory bytes: every array element read or written once (index arrays included, SELL padding
// and the second visit of a face from its other cell excluded).
double AlgoBytes::gradient(int nf) const {
  return C * (48.0 + 24.0 + 8.0 * nf + 24.0 * nf) + nnzOff * 8.0 + 4.0 * (C + 1) + Fb * (4.0 + 1.0 + 24.0 + 8.0 * nf);
}
double AlgoBytes::momentum() const {
  return C * (8.0 + 24 + 24 + 96 + 8 + 24 + 8) + Fi * 65.0 + nnzOff * 16.0 + 4.0 * (C + 1) + Fb * (80.0 + 1 + 24 + 4);
}
double AlgoBytes::pressure_rc() const {
  return C * 96.0 + Fi * (65.0 + 8) + nnzOff * 16.0 + 4.0 * (C + 1) + Fb * (80.0 + 1 + 24 + 8 + 4);
}
double AlgoBytes::nonorth() const { return C * 48.0 + Fi * 65.0 + nnzOff * 8.0 + 4.0 * (C + 1) + Fb * (80.0 + 1 + 4); }
double AlgoBytes::flux_final() const {
  return C * 136.0 + Fi * (65.0 + 16) + nnzOff * 8.0 + 4.0 * (C + 1) + Fb * (80.0 + 1 + 8 + 8 + 8 + 4);
}
double AlgoBytes::bicg_spmv(int nc) const { return 8.0 * C + 12.0 * nnzOff + 24.0 * nc * C; }
double AlgoBytes::pcg_spmv() const { return 40.0 * C + 12.0 * nnzOff; }

template <int WM>
static void lsq_grad_w(const LaunchCfg& lc, const DMesh& m, const GradArgs& a) {
  if (a.nf == 4) k_lsq_grad<4, WM><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
  else if (a.nf == 3) k_lsq_grad<3, WM><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
  else if (a.nf == 2) k_lsq_grad<2, WM><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
  else k_lsq_grad<1, WM><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
}
void launch_lsq_grad(const LaunchCfg& lc, const DMesh& m, const GradArgs& a) {
  ProfScope ps(lc, kKfGradient, lc.ab ? lc.ab->gradient(a.nf) : 0.0);
  const int wc = launch_width_class(m.maxW);
  if (wc == 4) lsq_grad_w<4>(lc, m, a);
  else if (wc == 6) lsq_grad_w<6>(lc, m, a);
  else if (wc == 8) lsq_grad_w<8>(lc, m, a);
  else lsq_grad_w<0>(lc, m, a);
}
template <class M>
void launch_momentum(const LaunchCfg& lc, const DMesh& m, const MomArgsT<M>& a) {
  ProfScope ps(lc, kKfMomentum, lc.ab ? lc.ab->momentum() : 0.0);
  with_width(m.maxW, [&](auto W) { launch_rows(lc, lc.rowBlocks, k_momentum<M, W.value>, m, a); });
}
template <class M>
void launch_pressure_rc(const LaunchCfg& lc, const DMesh& m, const PresArgsT<M>& a) {
  ProfScope ps(lc, kKfPressureRc, lc.ab ? lc.ab->pressure_rc() : 0.0);
  launch_rows(lc, lc.rowBlocks, k_pressure_rc<M>, m, a);
}
template void launch_momentum<double>(const LaunchCfg&, const DMesh&, const MomArgsT<double>&);
template void launch_momentum<float>(const LaunchCfg&, const DMesh&, const MomArgsT<float>&);
template void launch_pressure_rc<double>(const LaunchCfg&, const DMesh&, const PresArgsT<double>&);
template void launch_pressure_rc<float>(const LaunchCfg&, const DMesh&, const PresArgsT<float>&);
void launch_nonorth_rhs(const LaunchCfg& lc, const DMesh& m, const NonOrthArgs& a) {
  ProfScope ps(lc, kKfNonOrth, lc.ab ? lc.ab->nonorth() : 0.0);
  with_width(m.maxW, [&](auto W) { launch_rows(lc, lc.rowBlocks, k_nonorth_rhs<W.value>, m, a); });
}
void launch_flux_final(const LaunchCfg& lc, const DMesh& m, const FluxArgs& a) {
  const char* form = std::getenv("ANB_FLUX_FORM");  // "face": the face-parallel form (once per step)
  const bool faceForm = form && std::string(form) == "face";
  const int wc = launch_width_class(m.maxW);
  if (faceForm) {
    ProfScope ps(lc, kKfFluxFinal, lc.ab ? lc.ab->flux_final() : 0.0, 2);
    k_flux_faces<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
    if (wc == 4) k_flux_cells<4><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
    else if (wc == 6) k_flux_cells<6><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
    else if (wc == 8) k_flux_cells<8><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
    else k_flux_cells<0><<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
    return;
  }
  ProfScope ps(lc, kKfFluxFinal, lc.ab ? lc.ab->flux_final() : 0.0);
  // rows of six slots run the 8-slot instantiation: measured 197 against 311 us per launch on the
  // 970k-cell hex mesh (same registers and DRAM bytes; the 6-slot code waits longer on its loads)
  if (wc == 4) launch_rows(lc, lc.rowBlocks, k_flux_final<4>, m, a);
  else if (wc == 6 || wc == 8) launch_rows(lc, lc.rowBlocks, k_flux_final<8>, m, a);
  else launch_rows(lc, lc.rowBlocks, k_flux_final<0>, m, a);
}
void launch_patch_force(cudaStream_t s, const DMesh& m, int b0, int b1, int sign, double mu, const double* bA,
                        const double* bN, const double* U, const double* P, double* out) {
  g_launches += 1;
  k_patch_force<<<1, 512, 0, s>>>(m, b0, b1, sign, mu, bA, bN, U, P, out);
}

}  // namespace anb
