// Scalar elliptic and steady scalar-transport systems (sm_100a): the reference's libpoisson
// (libpoisson/src/{gradient,scalar_elliptic}.cu) and libscalar
// (libscalar/src/scalar_transport_library.cu) assemblies on the SIMPLE layout.
//
// Both kernels are cell-centric gathers like the SIMPLE face kernels: thread r owns row r, walks
// its SELL-32 slots (one per neighbour, each naming the connecting internal face) and its boundary
// faces.  The face loops of the reference scatter into four CSR slots per face; here each row
// accumulates its own diagonal and right-hand side, and writes its own off-diagonals.
#include "kernels.cuh"

namespace anb {

namespace {

// LSQ gradient with the scalar libraries' boundary rule (libpoisson/src/gradient.cu:21-83):
// Dirichlet faces constrain phi at the face centre; every other boundary face is the pure-normal
// constraint r = dn n, dphi = g dn with dn = max((x_f - x_P).n, 1e-30).
__global__ void __launch_bounds__(kBlock) k_scalar_grad(DMesh m, ScalarArgs a) {
  const int C = m.nCells;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    const double xr0 = m.cc[3 * r], xr1 = m.cc[3 * r + 1], xr2 = m.cc[3 * r + 2];
    const double pr = a.phi[r];
    double b0 = 0.0, b1 = 0.0, b2 = 0.0;
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      if (__ldg(&m.slotFace[e]) < 0) break;
      const int c = __ldg(&m.col[e]);
      const double r0 = __ldg(&m.cc[3 * c]) - xr0, r1 = __ldg(&m.cc[3 * c + 1]) - xr1, r2 = __ldg(&m.cc[3 * c + 2]) - xr2;
      const double w = 1.0 / fmax(r0 * r0 + r1 * r1 + r2 * r2, 1e-30);
      const double dp = w * (a.phi[c] - pr);
      b0 += r0 * dp;
      b1 += r1 * dp;
      b2 += r2 * dp;
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      const double* dd = m.bnd[bf].d;
      double r0 = dd[0], r1 = dd[1], r2 = dd[2], dphi;
      if (__ldg(&a.bcType[bf]) == kScalarDirichlet) {
        dphi = a.bcVal[bf] - pr;
      } else {
        const double n0 = a.bN[3 * bf], n1 = a.bN[3 * bf + 1], n2 = a.bN[3 * bf + 2];
        const double dn = fmax(r0 * n0 + r1 * n1 + r2 * n2, 1e-30);
        r0 = dn * n0;
        r1 = dn * n1;
        r2 = dn * n2;
        dphi = a.bcVal[bf] * dn;
      }
      const double w = 1.0 / fmax(r0 * r0 + r1 * r1 + r2 * r2, 1e-30);
      const double dp = w * dphi;
      b0 += r0 * dp;
      b1 += r1 * dp;
      b2 += r2 * dp;
    }
    const double* M = a.minv + 6 * r;
    a.g[r] = M[0] * b0 + M[1] * b1 + M[2] * b2;
    a.g[C + r] = M[1] * b0 + M[3] * b1 + M[4] * b2;
    a.g[2 * C + r] = M[2] * b0 + M[4] * b1 + M[5] * b2;
  }
}

// System assembly.  Elliptic: libpoisson/src/scalar_elliptic.cu:60-136, D = gamma |S|^2 / (d.S)
// per face, Dirichlet diag += D and rhs += D phi_b, Neumann rhs -= gamma g A, non-orthogonal
// rhs gamma T.grad_f with T = S - (D/gamma) d.  Transport: scalar_transport_library.cu:250-357,
// the same diffusion plus central (lambda-weighted) or upwind convection of the given face flux,
// -Sp V on the diagonal, Dirichlet rhs -= F phi_b, other boundaries diag += F and
// rhs += gamma g_n A.  The reference cell (scalar_elliptic.cu:126-135) fixes one row to its
// value; here its column is also moved to the right-hand side of the other rows, which keeps the
// matrix symmetric for CG and leaves the solution unchanged.
__global__ void __launch_bounds__(kBlock) k_scalar_assemble(DMesh m, ScalarArgs a) {
  const int C = m.nCells, nI = m.nInternal;
  const double* G = a.grad;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < C; r += gridDim.x * blockDim.x) {
    const double V = m.vol[r];
    double dg = a.sp ? -a.sp[r] * V : 0.0;
    double rh = a.src[r] * V;
    const bool isRef = (r == a.refCell);
    int W;
    const int base = row_base(m, r, W);
    for (int k = 0; k < W; ++k) {
      const int e = base + (k << 5);
      const int f = __ldg(&m.slotFace[e]);
      if (f < 0) {
        a.val[e] = 0.0;
        continue;
      }
      const int c = __ldg(&m.col[e]);
      const bool own = r < c;
      double lam, g, t[3], d[3];
      load_face(m.face, f, lam, g, t, d);
      const double S0 = t[0] + g * d[0], S1 = t[1] + g * d[1], S2 = t[2] + g * d[2];
      const double gam = a.gammaF[f];
      const double dS = d[0] * S0 + d[1] * S1 + d[2] * S2;
      const double D = gam * (S0 * S0 + S1 * S1 + S2 * S2) / fmax(dS, 1e-30);
      double off = -D;
      dg += D;
      if (a.flux) {
        const double F = a.flux[f];
        if (!a.upwind) {
          if (own) {
            dg += F * (1.0 - lam);
            off += F * lam;
          } else {
            off -= F * (1.0 - lam);
            dg -= F * lam;
          }
        } else if (own) {
          if (F >= 0.0) dg += F;
          else off += F;
        } else {
          if (F >= 0.0) off -= F;
          else dg -= F;
        }
      }
      if (a.nonorth) {
        const double Dg = D / fmax(gam, 1e-30);
        const double T0 = S0 - Dg * d[0], T1 = S1 - Dg * d[1], T2 = S2 - Dg * d[2];
        const int P = own ? r : c, N = own ? c : r;
        const double l1 = 1.0 - lam;
        const double gx = l1 * G[P] + lam * G[N], gy = l1 * G[C + P] + lam * G[C + N],
                     gz = l1 * G[2 * C + P] + lam * G[2 * C + N];
        const double corr = gam * (T0 * gx + T1 * gy + T2 * gz);
        rh += own ? corr : -corr;
      }
      if (c == a.refCell && !isRef) {
        rh -= off * a.refValue;
        off = 0.0;
      }
      a.val[e] = isRef ? 0.0 : off;
    }
    const int j0 = __ldg(&m.cbOff[r]), j1 = __ldg(&m.cbOff[r + 1]);
    for (int j = j0; j < j1; ++j) {
      const int bf = __ldg(&m.cbList[j]);
      double g, t[3], S[3], d[3];
      load_bnd(m.bnd, bf, g, t, S, d);
      const double gam = a.gammaF[nI + bf];
      const double dS = d[0] * S[0] + d[1] * S[1] + d[2] * S[2];
      const double D = gam * (S[0] * S[0] + S[1] * S[1] + S[2] * S[2]) / fmax(dS, 1e-30);
      const unsigned ty = __ldg(&a.bcType[bf]);
      const double v = a.bcVal[bf];
      const double F = a.flux ? a.flux[nI + bf] : 0.0;
      if (ty == kScalarDirichlet) {
        dg += D;
        rh += D * v;
        if (a.nonorth) {
          const double Dg = D / fmax(gam, 1e-30);
          const double T0 = S[0] - Dg * d[0], T1 = S[1] - Dg * d[1], T2 = S[2] - Dg * d[2];
          rh += gam * (T0 * G[r] + T1 * G[C + r] + T2 * G[2 * C + r]);
        }
        if (a.transport) rh += -F * v;
      } else if (a.transport) {
        const double gn = (ty == kScalarZeroGradient) ? 0.0 : v;
        rh += gam * gn * a.bA[bf];
        dg += F;
      } else {
        rh += -gam * v * a.bA[bf];
      }
    }
    if (isRef) {
      dg = 1.0;
      rh = a.refValue;
    }
    a.diag[r] = dg;
    a.rhs[r] = rh;
    if (a.wdinv) a.wdinv[r] = a.omega / dg;
  }
}

}  // namespace

void launch_scalar_grad(const LaunchCfg& lc, const DMesh& m, const ScalarArgs& a) {
  ProfScope ps(lc, kKfNone, 0.0);
  k_scalar_grad<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
}

void launch_scalar_assemble(const LaunchCfg& lc, const DMesh& m, const ScalarArgs& a) {
  ProfScope ps(lc, kKfNone, 0.0);
  k_scalar_assemble<<<lc.rowBlocks, kBlock, 0, lc.stream>>>(m, a);
}

}  // namespace anb
