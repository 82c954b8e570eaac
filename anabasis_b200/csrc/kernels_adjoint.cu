// Steady residual of the SIMPLE fixed point, its tangent (J v) and its adjoint (J^T w), for the
// discrete adjoint of the patch force (sm_100a).  No counterpart in the reference: the reference
// has no sensitivity code; the residual restates what its SIMPLE iteration converges to.
//
// At a converged SIMPLE state (main.cu:3388-3634) p' = 0 and U* = U, so the relaxation terms of
// the momentum system cancel and the state X = (U, p) satisfies
//   R_q[P] = sum_f s_Pf M_q^f + sum_b B_q^b + V_P (grad p)_q[P] = 0          (q = u, v, w)
//   R_c[P] = sum_f s_Pf phi_f + sum_b phi_b = 0
// with, per internal face f (owner o, neighbour n, s_Pf = +1 at o, -1 at n):
//   M_q^f = alpha (U_q[o] - U_q[n]) + F ubar_q - mu (grad U_q)_f . t        (faces with n.d > 1e-14)
//   phi_f = F - rho g rAU_f ((p[n] - p[o]) - (grad p)_f . d)                 (every internal face)
//   alpha = mu g, ubar = (1-lam) U[o] + lam U[n], F = rho ubar . S, (.)_f lam-interpolated,
//   rAU_P = V_P / (aP_P / uRelax), aP_P = sum_f (alpha + c_Pf F) + sum_b D_b, c = 1-lam at o, -lam at n
// and per boundary face b of P (momentum terms only where n.d_b > 1e-14):
//   u_b,q = BC value g_q if q is Dirichlet there, else U_q[P];  F_b = rho u_b . S_b
//   D_b = alpha_b if u is Dirichlet (the matrix carries the u types), else F_b
//   B_q^b = D_b U_q[P] - [Dir_q] (alpha_b g_q + mu (grad U_q)[P] . t_b - F_b g_q)
//   phi_b = F_b
// These are the terms of main.cu:1678-1896 (momentum, K25-K10) and 1474-1536 (Rhie-Chow K14,
// continuity K15), i.e. of k_momentum and k_pressure_rc.  Parameters: the Dirichlet velocity
// values of the parameter faces (the inlet) and mu.
//
// Every kernel is a cell-centric gather over the SELL-32 slots and the cell's boundary faces;
// face terms needed by both cells of a face are recomputed by each, so there are no atomics.
#include "kernels.cuh"

namespace anb {

namespace {

__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// interpolated gradient of field q (3*nCells SoA block) at a face
__device__ __forceinline__ void gface(const double* G, int C, int o, int n, double lam, double out[3]) {
  const double l1 = 1.0 - lam;
  out[0] = l1 * G[o] + lam * G[n];
  out[1] = l1 * G[C + o] + lam * G[C + n];
  out[2] = l1 * G[2 * C + o] + lam * G[2 * C + n];
}

// aP (unrelaxed momentum diagonal) and rAU of every cell.
__global__ void __launch_bounds__(kBlock) k_adj_base(DMesh m, AdjArgs a) {
  const int C = m.nCells;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double aP = 0.0;
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) continue;
      if (!(__ldg(&m.fFlags[f]) & 1)) continue;
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      double lam, g, t[3], d[3];
      load_face(m.face, f, lam, g, t, d);
      const int o = own ? r : c, n = own ? c : r;
      const double S[3] = {t[0] + g * d[0], t[1] + g * d[1], t[2] + g * d[2]};
      const double l1 = 1.0 - lam;
      const double ub[3] = {l1 * a.U[o] + lam * a.U[n], l1 * a.U[C + o] + lam * a.U[C + n],
                            l1 * a.U[2 * C + o] + lam * a.U[2 * C + n]};
      const double F = a.rho * dot3(ub, S);
      aP += a.mu * g + (own ? l1 : -lam) * F;
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      if (!(__ldg(&m.bFlags[bf]) & 1)) continue;
      double g, t[3], S[3], d[3];
      load_bnd(m.bnd, bf, g, t, S, d);
      const unsigned ty = __ldg(&m.bType[bf]);
      if (ty & 1u) {
        aP += a.mu * g;
      } else {
        double ubv[3];
        for (int q = 0; q < 3; ++q) ubv[q] = (ty & (1u << q)) ? m.bVal[q * m.nBoundary + bf] : a.U[q * C + r];
        aP += a.rho * dot3(ubv, S);
      }
    }
    const double diagR = a.relax ? aP * (1.0 / a.uRelax) : aP;
    a.aP[r] = aP;
    a.rau[r] = fabs(diagR) > 1e-30 ? m.vol[r] / diagR : 0.0;
  }
}

// Steady residual R (4 x nCells: u | v | w | continuity); G = gradients of u, v, w, p (12C).
__global__ void __launch_bounds__(kBlock) k_adj_residual(DMesh m, AdjArgs a, double* R) {
  const int C = m.nCells;
  const double* G = a.G;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    const double V = m.vol[r];
    double Rq[3] = {V * G[9 * C + r], V * G[10 * C + r], V * G[11 * C + r]};
    double Rc = 0.0;
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) continue;
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      const double s = own ? 1.0 : -1.0;
      double lam, g, t[3], d[3];
      load_face(m.face, f, lam, g, t, d);
      const int o = own ? r : c, n = own ? c : r;
      const double S[3] = {t[0] + g * d[0], t[1] + g * d[1], t[2] + g * d[2]};
      const double l1 = 1.0 - lam;
      double ub[3];
      for (int q = 0; q < 3; ++q) ub[q] = l1 * a.U[q * C + o] + lam * a.U[q * C + n];
      const double F = a.rho * dot3(ub, S);
      if (__ldg(&m.fFlags[f]) & 1) {
        const double alpha = a.mu * g;
        for (int q = 0; q < 3; ++q) {
          double gf[3];
          gface(G + 3 * q * C, C, o, n, lam, gf);
          Rq[q] += s * (alpha * (a.U[q * C + o] - a.U[q * C + n]) + F * ub[q] - a.mu * dot3(gf, t));
        }
      }
      double gp[3];
      gface(G + 9 * C, C, o, n, lam, gp);
      const double rAUf = l1 * a.rau[o] + lam * a.rau[n];
      Rc += s * (F - a.rho * g * rAUf * ((a.P[n] - a.P[o]) - dot3(gp, d)));
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      double g, t[3], S[3], d[3];
      load_bnd(m.bnd, bf, g, t, S, d);
      const unsigned ty = __ldg(&m.bType[bf]);
      double ubv[3];
      for (int q = 0; q < 3; ++q) ubv[q] = (ty & (1u << q)) ? m.bVal[q * m.nBoundary + bf] : a.U[q * C + r];
      const double Fb = a.rho * dot3(ubv, S);
      Rc += Fb;
      if (!(__ldg(&m.bFlags[bf]) & 1)) continue;
      const double alpha = a.mu * g;
      const double Db = (ty & 1u) ? alpha : Fb;
      for (int q = 0; q < 3; ++q) {
        Rq[q] += Db * a.U[q * C + r];
        if (ty & (1u << q)) {
          const double gq = ubv[q];
          const double gt = G[3 * q * C + r] * t[0] + G[3 * q * C + C + r] * t[1] + G[3 * q * C + 2 * C + r] * t[2];
          Rq[q] -= alpha * gq + a.mu * gt - Fb * gq;
        }
      }
    }
    R[r] = Rq[0];
    R[C + r] = Rq[1];
    R[2 * C + r] = Rq[2];
    R[3 * C + r] = Rc;
  }
}

// ---- tangent ---------------------------------------------------------------------------------
// daP of every cell for the tangent (dU, dg, dmu).
__global__ void __launch_bounds__(kBlock) k_jvp_ap(DMesh m, AdjArgs a, TanArgs t_) {
  const int C = m.nCells;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double daP = 0.0;
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) continue;
      if (!(__ldg(&m.fFlags[f]) & 1)) continue;
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      double lam, g, t[3], d[3];
      load_face(m.face, f, lam, g, t, d);
      const int o = own ? r : c, n = own ? c : r;
      const double S[3] = {t[0] + g * d[0], t[1] + g * d[1], t[2] + g * d[2]};
      const double l1 = 1.0 - lam;
      double dub[3];
      for (int q = 0; q < 3; ++q) dub[q] = l1 * t_.dU[q * C + o] + lam * t_.dU[q * C + n];
      daP += t_.dmu * g + (own ? l1 : -lam) * a.rho * dot3(dub, S);
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      if (!(__ldg(&m.bFlags[bf]) & 1)) continue;
      double g, t[3], S[3], d[3];
      load_bnd(m.bnd, bf, g, t, S, d);
      const unsigned ty = __ldg(&m.bType[bf]);
      if (ty & 1u) {
        daP += t_.dmu * g;
      } else {
        double dub[3];
        for (int q = 0; q < 3; ++q) dub[q] = (ty & (1u << q)) ? t_.dg[q * m.nBoundary + bf] : t_.dU[q * C + r];
        daP += a.rho * dot3(dub, S);
      }
    }
    t_.daP[r] = daP;
  }
}

// dR = J (dU, dp) + R_theta (dg, dmu); dG = gradients of du, dv, dw (BC values dg) and dp.
__global__ void __launch_bounds__(kBlock) k_jvp(DMesh m, AdjArgs a, TanArgs t_, double* dR) {
  const int C = m.nCells;
  const double* G = a.G;
  const double* dG = t_.dG;
  const double dmu = t_.dmu;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    const double V = m.vol[r];
    double Rq[3] = {V * dG[9 * C + r], V * dG[10 * C + r], V * dG[11 * C + r]};
    double Rc = 0.0;
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) continue;
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      const double s = own ? 1.0 : -1.0;
      double lam, g, t[3], d[3];
      load_face(m.face, f, lam, g, t, d);
      const int o = own ? r : c, n = own ? c : r;
      const double S[3] = {t[0] + g * d[0], t[1] + g * d[1], t[2] + g * d[2]};
      const double l1 = 1.0 - lam;
      double ub[3], dub[3];
      for (int q = 0; q < 3; ++q) {
        ub[q] = l1 * a.U[q * C + o] + lam * a.U[q * C + n];
        dub[q] = l1 * t_.dU[q * C + o] + lam * t_.dU[q * C + n];
      }
      const double F = a.rho * dot3(ub, S), dF = a.rho * dot3(dub, S);
      if (__ldg(&m.fFlags[f]) & 1) {
        const double alpha = a.mu * g, dalpha = dmu * g;
        for (int q = 0; q < 3; ++q) {
          double gf[3], dgf[3];
          gface(G + 3 * q * C, C, o, n, lam, gf);
          gface(dG + 3 * q * C, C, o, n, lam, dgf);
          const double dM = dalpha * (a.U[q * C + o] - a.U[q * C + n]) +
                            alpha * (t_.dU[q * C + o] - t_.dU[q * C + n]) + dF * ub[q] + F * dub[q] -
                            dmu * dot3(gf, t) - a.mu * dot3(dgf, t);
          Rq[q] += s * dM;
        }
      }
      double gp[3], dgp[3];
      gface(G + 9 * C, C, o, n, lam, gp);
      gface(dG + 9 * C, C, o, n, lam, dgp);
      const double rAUf = l1 * a.rau[o] + lam * a.rau[n];
      const double drau_o = a.aP[o] != 0.0 ? -a.rau[o] * t_.daP[o] / a.aP[o] : 0.0;
      const double drau_n = a.aP[n] != 0.0 ? -a.rau[n] * t_.daP[n] / a.aP[n] : 0.0;
      const double drAUf = l1 * drau_o + lam * drau_n;
      const double X = (a.P[n] - a.P[o]) - dot3(gp, d);
      const double dX = (t_.dp[n] - t_.dp[o]) - dot3(dgp, d);
      Rc += s * (dF - a.rho * g * (drAUf * X + rAUf * dX));
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      double g, t[3], S[3], d[3];
      load_bnd(m.bnd, bf, g, t, S, d);
      const unsigned ty = __ldg(&m.bType[bf]);
      double ubv[3], dubv[3];
      for (int q = 0; q < 3; ++q) {
        const bool dir = ty & (1u << q);
        ubv[q] = dir ? m.bVal[q * m.nBoundary + bf] : a.U[q * C + r];
        dubv[q] = dir ? t_.dg[q * m.nBoundary + bf] : t_.dU[q * C + r];
      }
      const double Fb = a.rho * dot3(ubv, S), dFb = a.rho * dot3(dubv, S);
      Rc += dFb;
      if (!(__ldg(&m.bFlags[bf]) & 1)) continue;
      const double alpha = a.mu * g, dalpha = dmu * g;
      const double Db = (ty & 1u) ? alpha : Fb, dDb = (ty & 1u) ? dalpha : dFb;
      for (int q = 0; q < 3; ++q) {
        Rq[q] += dDb * a.U[q * C + r] + Db * t_.dU[q * C + r];
        if (ty & (1u << q)) {
          const double gq = ubv[q], dgq = dubv[q];
          const double* Gq = G + 3 * q * C;
          const double* dGq = dG + 3 * q * C;
          const double gt = Gq[r] * t[0] + Gq[C + r] * t[1] + Gq[2 * C + r] * t[2];
          const double dgt = dGq[r] * t[0] + dGq[C + r] * t[1] + dGq[2 * C + r] * t[2];
          Rq[q] -= dalpha * gq + alpha * dgq + dmu * gt + a.mu * dgt - dFb * gq - Fb * dgq;
        }
      }
    }
    dR[r] = Rq[0];
    dR[C + r] = Rq[1];
    dR[2 * C + r] = Rq[2];
    dR[3 * C + r] = Rc;
  }
}

// ---- adjoint ---------------------------------------------------------------------------------
// Pass A: per cell the adjoint of aP (abar) and h = Minv * (adjoint of each gradient), for the
// gradients of u, v, w (momentum non-orthogonal terms) and p (Rhie-Chow and the pressure source).
__global__ void __launch_bounds__(kBlock) k_vjp_a(DMesh m, AdjArgs a, AdjWork w_) {
  const int C = m.nCells;
  const double* w = w_.w;
  const double* wc = w + 3 * C;
  const double* G = a.G;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    const double V = m.vol[r];
    double Gb[4][3];
    for (int q = 0; q < 3; ++q) {
      Gb[q][0] = Gb[q][1] = Gb[q][2] = 0.0;
      Gb[3][q] = V * w[q * C + r];
    }
    double rauBar = 0.0;
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) continue;
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      double lam, g, t[3], d[3];
      load_face(m.face, f, lam, g, t, d);
      const int o = own ? r : c, n = own ? c : r;
      const double cw = own ? 1.0 - lam : lam;  // interpolation weight of this cell
      if (__ldg(&m.fFlags[f]) & 1) {
        for (int q = 0; q < 3; ++q) {
          const double wt = w[q * C + o] - w[q * C + n];
          for (int k2 = 0; k2 < 3; ++k2) Gb[q][k2] -= a.mu * cw * t[k2] * wt;
        }
      }
      const double wtc = wc[o] - wc[n];
      double gp[3];
      gface(G + 9 * C, C, o, n, lam, gp);
      const double rAUf = (1.0 - lam) * a.rau[o] + lam * a.rau[n];
      const double X = (a.P[n] - a.P[o]) - dot3(gp, d);
      rauBar -= a.rho * g * X * cw * wtc;
      for (int k2 = 0; k2 < 3; ++k2) Gb[3][k2] += a.rho * g * rAUf * cw * d[k2] * wtc;
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      if (!(__ldg(&m.bFlags[bf]) & 1)) continue;
      const unsigned ty = __ldg(&m.bType[bf]);
      const double* tb = m.bnd[bf].t;
      for (int q = 0; q < 3; ++q)
        if (ty & (1u << q))
          for (int k2 = 0; k2 < 3; ++k2) Gb[q][k2] -= w[q * C + r] * a.mu * tb[k2];
    }
    w_.abar[r] = a.aP[r] != 0.0 ? -a.rau[r] / a.aP[r] * rauBar : 0.0;
    const double* M = m.minv + 6 * r;
    for (int q = 0; q < 4; ++q) {
      double* h = w_.h + 3 * q * C;
      h[r] = M[0] * Gb[q][0] + M[1] * Gb[q][1] + M[2] * Gb[q][2];
      h[C + r] = M[1] * Gb[q][0] + M[3] * Gb[q][1] + M[4] * Gb[q][2];
      h[2 * C + r] = M[2] * Gb[q][0] + M[4] * Gb[q][1] + M[5] * Gb[q][2];
    }
  }
}

// LSQ-gradient transpose at cell r for field q: sum over neighbours Y of w (x_r - x_Y).h[Y]
// minus (sum over neighbours of w (x_Y - x_r) + Dirichlet faces w_b d_b) . h[r].
__device__ __forceinline__ double grad_transpose(const DMesh& m, int r, int base, int W, const double* h, int C,
                                                 unsigned dirBit) {
  const double xr[3] = {m.cc[3 * r], m.cc[3 * r + 1], m.cc[3 * r + 2]};
  const double hr[3] = {h[r], h[C + r], h[2 * C + r]};
  double out = 0.0;
  for (int k = 0; k < W; ++k) {
    const int e = base + (k << 5);
    if (__ldg(&m.slotFace[e]) < 0) break;
    const int c = __ldg(&m.col[e]);
    const double rr[3] = {__ldg(&m.cc[3 * c]) - xr[0], __ldg(&m.cc[3 * c + 1]) - xr[1], __ldg(&m.cc[3 * c + 2]) - xr[2]};
    const double w = 1.0 / fmax(dot3(rr, rr), 1e-30);
    // neighbour c's gradient uses w (x_r - x_c) (phi_r - phi_c): coefficient of phi_r is +w(x_r - x_c)
    out += w * (-(rr[0] * h[c] + rr[1] * h[C + c] + rr[2] * h[2 * C + c]));
    // own gradient: coefficient of phi_r is -w (x_c - x_r)
    out -= w * dot3(rr, hr);
  }
  const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
  for (int j = j0; j < j1; ++j) {
    const int bf = __ldg(&m.cbList[j]);
    if (!(__ldg(&m.bType[bf]) & dirBit)) continue;
    const double* dd = m.bnd[bf].d;
    const double w = 1.0 / fmax(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2], 1e-30);
    out -= w * dot3(dd, hr);
  }
  return out;
}

// Pass B: (Ubar, pbar) = J^T w, the parameter adjoints gbar (per boundary face, 3 components)
// and the partial sums of mubar (reduced in the last block into w_.muBar[0]).
__global__ void __launch_bounds__(kBlock) k_vjp_b(DMesh m, AdjArgs a, AdjWork w_, double* out) {
  __shared__ double sm[32];
  const int C = m.nCells;
  const double* w = w_.w;
  const double* wc = w + 3 * C;
  const double* G = a.G;
  const double* h = w_.h;
  const double* ab = w_.abar;
  const double rho = a.rho, mu = a.mu;
  double muAcc[1] = {0.0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double Ub[3] = {0.0, 0.0, 0.0}, pb = 0.0;
    double gSum = 0.0;  // sum of g over the momentum faces of r (mu dependence of aP)
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) continue;
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      const double s = own ? 1.0 : -1.0;
      double lam, g, t[3], d[3];
      load_face(m.face, f, lam, g, t, d);
      const int o = own ? r : c, n = own ? c : r;
      const double S[3] = {t[0] + g * d[0], t[1] + g * d[1], t[2] + g * d[2]};
      const double l1 = 1.0 - lam;
      const double cw = own ? l1 : lam;
      double ub[3];
      for (int q = 0; q < 3; ++q) ub[q] = l1 * a.U[q * C + o] + lam * a.U[q * C + n];
      const double F = rho * dot3(ub, S);
      const double wtc = wc[o] - wc[n];
      double Fbar = wtc;  // continuity flux
      if (__ldg(&m.fFlags[f]) & 1) {
        const double alpha = mu * g;
        double zeta = 0.0;
        for (int q = 0; q < 3; ++q) {
          const double wt = w[q * C + o] - w[q * C + n];
          Ub[q] += s * alpha * wt + F * cw * wt;
          zeta += ub[q] * wt;
          if (own) {
            double gf[3];
            gface(G + 3 * q * C, C, o, n, lam, gf);
            muAcc[0] += wt * (g * (a.U[q * C + o] - a.U[q * C + n]) - dot3(gf, t));
          }
        }
        Fbar += zeta + l1 * ab[o] - lam * ab[n];
        gSum += g;
      }
      for (int q = 0; q < 3; ++q) Ub[q] += rho * S[q] * cw * Fbar;
      const double rAUf = l1 * a.rau[o] + lam * a.rau[n];
      pb += s * rho * g * rAUf * wtc;
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      double g, t[3], S[3], d[3];
      load_bnd(m.bnd, bf, g, t, S, d);
      const unsigned ty = __ldg(&m.bType[bf]);
      double ubv[3], gbar[3] = {0.0, 0.0, 0.0};
      for (int q = 0; q < 3; ++q) ubv[q] = (ty & (1u << q)) ? m.bVal[q * m.nBoundary + bf] : a.U[q * C + r];
      const double Fb = rho * dot3(ubv, S);
      double FbBar = wc[r];  // continuity flux
      if (__ldg(&m.bFlags[bf]) & 1) {
        const double alpha = mu * g;
        const double Db = (ty & 1u) ? alpha : Fb;
        double eta = 0.0, xi = 0.0;
        for (int q = 0; q < 3; ++q) {
          const double wq = w[q * C + r];
          eta += wq * a.U[q * C + r];
          Ub[q] += Db * wq;
          if (ty & (1u << q)) {
            const double kap = -wq, gq = ubv[q];
            const double* Gq = G + 3 * q * C;
            const double gt = Gq[r] * t[0] + Gq[C + r] * t[1] + Gq[2 * C + r] * t[2];
            gbar[q] += kap * alpha - kap * Fb;
            xi -= kap * gq;
            muAcc[0] += kap * (g * gq + gt);
          }
        }
        FbBar += xi;
        if (ty & 1u) {
          muAcc[0] += eta * g;
          gSum += g;
        } else {
          FbBar += eta + ab[r];
        }
      }
      for (int q = 0; q < 3; ++q) {
        if (ty & (1u << q)) {
          gbar[q] += rho * S[q] * FbBar;
          // Dirichlet value in the LSQ gradient of component q: w_b d_b . h_q
          const double* hq = h + 3 * q * C;
          const double wb = 1.0 / fmax(d[0] * d[0] + d[1] * d[1] + d[2] * d[2], 1e-30);
          gbar[q] += wb * (d[0] * hq[r] + d[1] * hq[C + r] + d[2] * hq[2 * C + r]);
        } else {
          Ub[q] += rho * S[q] * FbBar;
        }
      }
      if (w_.gbar)
        for (int q = 0; q < 3; ++q) w_.gbar[q * m.nBoundary + bf] = gbar[q];
    }
    muAcc[0] += ab[r] * gSum;
    for (int q = 0; q < 3; ++q) Ub[q] += grad_transpose(m, r, base, W, h + 3 * q * C, C, 1u << q);
    pb += grad_transpose(m, r, base, W, h + 9 * C, C, 8u);
    out[r] = Ub[0];
    out[C + r] = Ub[1];
    out[2 * C + r] = Ub[2];
    out[3 * C + r] = pb;
  }
  if (grid_reduce<1>(muAcc, 0u, a.red, sm) && threadIdx.x == 0) w_.muBar[0] = muAcc[0];
}

// Objective J = dir . (patch force) and its derivative in (U, p) and mu, cell-centric over the
// patch faces [b0, b1) (the rule of k_patch_force).  out: 4C; val[0] = J, val[1] = dJ/dmu.
__global__ void __launch_bounds__(kBlock) k_obj_grad(DMesh m, AdjArgs a, ObjArgs ob, double* out) {
  __shared__ double sm[2 * 32];
  const int C = m.nCells;
  double acc[2] = {0.0, 0.0};
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double Ub[3] = {0.0, 0.0, 0.0}, pb = 0.0;
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int b = __ldg(&m.cbList[j]);
      if (b < ob.b0 || b >= ob.b1) continue;
      const double A = ob.bA[b];
      if (A <= 1.0e-300) continue;
      double n0 = (double)ob.sign * ob.bN[3 * b], n1 = (double)ob.sign * ob.bN[3 * b + 1],
             n2 = (double)ob.sign * ob.bN[3 * b + 2];
      const double nm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
      if (nm <= 1.0e-300) continue;
      const double inv = 1.0 / nm;
      n0 *= inv; n1 *= inv; n2 *= inv;
      const double* d = m.bnd[b].d;
      const double dx0 = -d[0], dx1 = -d[1], dx2 = -d[2];
      double dn = dx0 * n0 + dx1 * n1 + dx2 * n2;
      if (dn <= 1.0e-14) dn = fabs(dn);
      if (dn <= 1.0e-14) dn = sqrt(dx0 * dx0 + dx1 * dx1 + dx2 * dx2);
      if (dn <= 1.0e-14) continue;
      const double nn[3] = {n0, n1, n2};
      const double u[3] = {a.U[r], a.U[C + r], a.U[2 * C + r]};
      const double Un = dot3(u, nn);
      const double dirn = ob.dir[0] * n0 + ob.dir[1] * n1 + ob.dir[2] * n2;
      double dirt = 0.0;
      for (int q = 0; q < 3; ++q) {
        const double tq = u[q] - Un * nn[q];
        dirt += ob.dir[q] * tq;
        Ub[q] += a.mu * A / dn * (ob.dir[q] - dirn * nn[q]);
      }
      pb -= dirn * A;
      acc[0] += -a.P[r] * dirn * A + a.mu * dirt / dn * A;
      acc[1] += dirt / dn * A;
    }
    out[r] = Ub[0];
    out[C + r] = Ub[1];
    out[2 * C + r] = Ub[2];
    out[3 * C + r] = pb;
  }
  if (grid_reduce<2>(acc, 0u, a.red, sm) && threadIdx.x == 0) {
    ob.val[0] = acc[0];
    ob.val[1] = acc[1];
  }
}

// ---- preconditioner pieces --------------------------------------------------------------------
// y = D_U v: continuity of the interpolated velocity field v (boundary: non-Dirichlet comps)
__global__ void __launch_bounds__(kBlock) k_div_u(DMesh m, double rho, const double* v, double* y) {
  const int C = m.nCells;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double acc = 0.0;
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) continue;
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      double lam, g, t[3], d[3];
      load_face(m.face, f, lam, g, t, d);
      const int o = own ? r : c, n = own ? c : r;
      const double l1 = 1.0 - lam;
      double fl = 0.0;
      for (int q = 0; q < 3; ++q) fl += (t[q] + g * d[q]) * (l1 * v[q * C + o] + lam * v[q * C + n]);
      acc += (own ? 1.0 : -1.0) * rho * fl;
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      const unsigned ty = __ldg(&m.bType[bf]);
      const double* S = m.bnd[bf].S;
      for (int q = 0; q < 3; ++q)
        if (!(ty & (1u << q))) acc += rho * S[q] * v[q * C + r];
    }
    y[r] = acc;
  }
}

// Y = D_U^T w (3C)
__global__ void __launch_bounds__(kBlock) k_div_u_t(DMesh m, double rho, const double* w, double* Y) {
  const int C = m.nCells;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    double Ub[3] = {0.0, 0.0, 0.0};
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) continue;
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      double lam, g, t[3], d[3];
      load_face(m.face, f, lam, g, t, d);
      const int o = own ? r : c, n = own ? c : r;
      const double cw = own ? 1.0 - lam : lam;
      const double wt = w[o] - w[n];
      for (int q = 0; q < 3; ++q) Ub[q] += rho * (t[q] + g * d[q]) * cw * wt;
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      const unsigned ty = __ldg(&m.bType[bf]);
      const double* S = m.bnd[bf].S;
      for (int q = 0; q < 3; ++q)
        if (!(ty & (1u << q))) Ub[q] += rho * S[q] * w[r];
    }
    for (int q = 0; q < 3; ++q) Y[q * C + r] = Ub[q];
  }
}

// y = LSQ-gradient transpose of the 3-vector field s scaled per cell by fac*sc (h = Minv (fac sc s)),
// field with Dirichlet bit dirBit (two passes: h, then the gather)
__global__ void __launch_bounds__(kBlock) k_scaled_minv(DMesh m, const double* sc, double fac, const double* s,
                                                        double* h) {
  const int C = m.nCells;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    const double* M = m.minv + 6 * r;
    const double k = fac * (sc ? sc[r] : 1.0);
    const double g0 = k * s[r], g1 = k * s[C + r], g2 = k * s[2 * C + r];
    h[r] = M[0] * g0 + M[1] * g1 + M[2] * g2;
    h[C + r] = M[1] * g0 + M[3] * g1 + M[4] * g2;
    h[2 * C + r] = M[2] * g0 + M[4] * g1 + M[5] * g2;
  }
}
__global__ void __launch_bounds__(kBlock) k_grad_t(DMesh m, const double* h, unsigned dirBit, double* y) {
  const int C = m.nCells;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    int W;
    const int base = row_base(m, r, W);
    y[r] = grad_transpose(m, r, base, W, h, C, dirBit);
  }
}

// x_U -= fac * sc * grad(p) (3C), grad p given (3C SoA)
__global__ void __launch_bounds__(kBlock) k_sub_scaled_grad(int C, const double* sc, double fac, const double* gp,
                                                            double* x) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x)
    for (int q = 0; q < 3; ++q) x[q * C + r] -= fac * sc[r] * gp[q * C + r];
}

__global__ void __launch_bounds__(kBlock) k_permute(int n, const int* idx, const double* src, double* dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

// ---- vector kernels for the Krylov solver (deterministic: fixed partition, fixed order) ----
// partials[j * gridDim.x + block] = sum over the block's rows of V_j . x, j < k
__global__ void __launch_bounds__(kBlock) k_mdot_partial(size_t n, int k, const double* V, size_t ld, const double* x,
                                                         double* partials) {
  __shared__ double sm[32];
  for (int j = 0; j < k; ++j) {
    double v[1] = {0.0};
    const double* Vj = V + (size_t)j * ld;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
      v[0] += Vj[i] * x[i];
    block_reduce<1>(v, 0u, sm);
    if (threadIdx.x == 0) partials[(size_t)j * gridDim.x + blockIdx.x] = v[0];
  }
}
__global__ void k_mdot_final(int k, int nb, const double* partials, double* out) {
  __shared__ double sm[32];
  for (int j = 0; j < k; ++j) {
    double v[1] = {0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v[0] += partials[(size_t)j * nb + b];
    block_reduce<1>(v, 0u, sm);
    if (threadIdx.x == 0) out[j] = v[0];
  }
}
// x = beta x + sum_j coef[j] V_j
__global__ void __launch_bounds__(kBlock) k_lincomb(size_t n, int k, const double* V, size_t ld, const double* coef,
                                                    double beta, double* x) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double s = beta == 0.0 ? 0.0 : beta * x[i];
    for (int j = 0; j < k; ++j) s += coef[j] * V[(size_t)j * ld + i];
    x[i] = s;
  }
}

}  // namespace

static int blocks(const LaunchCfg& lc) { return lc.rowBlocks; }

void adj_base(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a) {
  g_launches += 1;
  k_adj_base<<<blocks(lc), kBlock, 0, lc.stream>>>(m, a);
}
void adj_residual(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a, double* R) {
  g_launches += 1;
  k_adj_residual<<<blocks(lc), kBlock, 0, lc.stream>>>(m, a, R);
}
void adj_jvp(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a, const TanArgs& t, double* dR) {
  g_launches += 2;
  k_jvp_ap<<<blocks(lc), kBlock, 0, lc.stream>>>(m, a, t);
  k_jvp<<<blocks(lc), kBlock, 0, lc.stream>>>(m, a, t, dR);
}
void adj_vjp(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a, const AdjWork& w, double* out) {
  g_launches += 2;
  k_vjp_a<<<blocks(lc), kBlock, 0, lc.stream>>>(m, a, w);
  k_vjp_b<<<blocks(lc), kBlock, 0, lc.stream>>>(m, a, w, out);
}
void adj_objective(const LaunchCfg& lc, const DMesh& m, const AdjArgs& a, const ObjArgs& o, double* out) {
  g_launches += 1;
  k_obj_grad<<<blocks(lc), kBlock, 0, lc.stream>>>(m, a, o, out);
}
void adj_div_u(const LaunchCfg& lc, const DMesh& m, double rho, const double* v, double* y) {
  g_launches += 1;
  k_div_u<<<blocks(lc), kBlock, 0, lc.stream>>>(m, rho, v, y);
}
void adj_div_u_t(const LaunchCfg& lc, const DMesh& m, double rho, const double* w, double* Y) {
  g_launches += 1;
  k_div_u_t<<<blocks(lc), kBlock, 0, lc.stream>>>(m, rho, w, Y);
}
void adj_grad_t(const LaunchCfg& lc, const DMesh& m, const double* sc, double fac, const double* s, double* h,
                unsigned dirBit, double* y) {
  g_launches += 2;
  k_scaled_minv<<<blocks(lc), kBlock, 0, lc.stream>>>(m, sc, fac, s, h);
  k_grad_t<<<blocks(lc), kBlock, 0, lc.stream>>>(m, h, dirBit, y);
}
void adj_sub_scaled_grad(const LaunchCfg& lc, int C, const double* sc, double fac, const double* gp, double* x) {
  g_launches += 1;
  k_sub_scaled_grad<<<blocks(lc), kBlock, 0, lc.stream>>>(C, sc, fac, gp, x);
}
void adj_permute(const LaunchCfg& lc, int n, const int* idx, const double* src, double* dst) {
  g_launches += 1;
  k_permute<<<blocks(lc), kBlock, 0, lc.stream>>>(n, idx, src, dst);
}
void vec_mdot(const LaunchCfg& lc, size_t n, int k, const double* V, size_t ld, const double* x, double* partials,
              double* out) {
  g_launches += 2;
  const int nb = blocks(lc);
  k_mdot_partial<<<nb, kBlock, 0, lc.stream>>>(n, k, V, ld, x, partials);
  k_mdot_final<<<1, 1024, 0, lc.stream>>>(k, nb, partials, out);
}
void vec_lincomb(const LaunchCfg& lc, size_t n, int k, const double* V, size_t ld, const double* coef, double beta,
                 double* x) {
  g_launches += 1;
  k_lincomb<<<blocks(lc), kBlock, 0, lc.stream>>>(n, k, V, ld, coef, beta, x);
}

}  // namespace anb
