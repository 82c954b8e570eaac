// Discrete adjoint and tangent-linear of the converged SIMPLE state (include/anb.h, "steady
// sensitivities").  No counterpart in the reference.
//
// The converged state X = (U, p) solves R(X; g, mu) = 0 (kernels_adjoint.cu).  For the objective
// J = dir . (patch force):
//   tangent-linear  J_X dX = -R_theta dtheta,  dJ = J_X . dX + J_mu dmu
//   adjoint         J_X^T lambda = (dJ/dX)^T,  dJ/dg = -R_g^T lambda,  dJ/dmu = J_mu - R_mu^T lambda
// Both linear systems are solved by right-preconditioned FGMRES whose operator products are the
// hand-written tangent / adjoint kernels, and whose preconditioner is one SIMPLE-type block
// sweep built from the forward solver's pieces: the momentum matrix at the converged state
// (BiCGSTAB with A, or with A^T for the adjoint), the continuity of the velocity (D_U, D_U^T),
// and the pressure matrix with its AMG hierarchy (PCG).  Only the converged state is kept (the
// coefficient arrays are recomputed from it), never the iteration history.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "context.hpp"

namespace anb {

struct AdjointData {
  DevArena ar;
  int C = 0, nB = 0, mBasis = 0;
  size_t N = 0;  // 4 * nCells
  double *aP = nullptr, *rau = nullptr, *G = nullptr, *dG = nullptr, *daP = nullptr;
  double *abar = nullptr, *h = nullptr, *gbar = nullptr, *dgZero = nullptr, *dgDir = nullptr, *zeroB = nullptr;
  double *muBar = nullptr, *objVal = nullptr, *partials = nullptr, *coef = nullptr;
  double *gX = nullptr, *R = nullptr, *t1 = nullptr, *t2 = nullptr, *t3 = nullptr, *xs = nullptr, *rhs = nullptr;
  double *V = nullptr, *Z = nullptr;  // FGMRES bases ((m+1) N, m N)
  double* valT = nullptr;
  int* twin = nullptr;
  bool precReady = false;
  // Preconditioner controls (ANB_ADJ_* environment variables override them).  The momentum
  // block uses the SIMPLE iteration's own relaxed matrix (diagonal aP/uRelax): Jacobi-BiCGSTAB
  // needs ~4 iterations on it against ~135 on the unrelaxed one, which made the adjoint 10x
  // slower at 1M cells.  The pressure block is the pressure matrix scaled by rho/uRelax: for smooth
  // pressure modes the Schur complement D_p - D_U A^-1 G is dominated by -D_U A^-1 G, which is
  // the rAU/uRelax-weighted Laplacian, while the Rhie-Chow part D_p acts on the oscillatory ones.
  int restart = 40;
  double rtol = 1e-10;  // relative tolerance of the tangent-linear and adjoint systems
  double momRtol = 1e-2, pRtol = 1e-2, schur = 1.0;
  int momMaxit = 200, momRelaxed = 1;
  long long momIts = 0, pIts = 0;  // inner iterations since the last reset
};

void adjoint_release(anb_ctx* c) {
  if (!c->adj) return;
  c->adj->ar.release();
  delete c->adj;
  c->adj = nullptr;
}

namespace {

constexpr int kMaxRestart = 120;

double env_or(const char* name, double dflt) {
  const char* v = std::getenv(name);
  return v ? std::atof(v) : dflt;
}

AdjointData& adj(anb_ctx* c) {
  if (c->adj) return *c->adj;
  auto* d = new AdjointData();
  c->adj = d;
  DevArena& A = d->ar;
  const int C = c->C;
  d->C = C;
  d->nB = c->nB;
  d->N = (size_t)4 * C;
  d->restart = std::max(4, std::min(kMaxRestart, (int)env_or("ANB_ADJ_RESTART", d->restart)));
  d->rtol = env_or("ANB_ADJ_RTOL", d->rtol);
  d->momRtol = env_or("ANB_ADJ_MOM_RTOL", d->momRtol);
  d->pRtol = env_or("ANB_ADJ_P_RTOL", d->pRtol);
  d->schur = env_or("ANB_ADJ_SCHUR", c->prm.u_relax < 0.999999 ? c->prm.u_relax : 1.0);
  d->momMaxit = (int)env_or("ANB_ADJ_MOM_MAXIT", d->momMaxit);
  d->momRelaxed = (int)env_or("ANB_ADJ_MOM_RELAXED", d->momRelaxed);
  d->mBasis = d->restart;
  d->aP = A.alloc<double>(C);
  d->rau = A.alloc<double>(C);
  d->G = A.alloc<double>((size_t)12 * C);
  d->dG = A.alloc<double>((size_t)12 * C);
  d->daP = A.alloc<double>(C);
  d->abar = A.alloc<double>(C);
  d->h = A.alloc<double>((size_t)12 * C);
  d->gbar = A.alloc<double>((size_t)3 * c->nB);
  d->dgZero = A.alloc<double>((size_t)3 * c->nB);
  d->dgDir = A.alloc<double>((size_t)3 * c->nB);
  d->zeroB = A.alloc<double>(c->nB);
  d->muBar = A.alloc<double>(2);
  d->objVal = A.alloc<double>(2);
  d->partials = A.alloc<double>((size_t)c->lc.rowBlocks * (d->mBasis + 2));
  d->coef = A.alloc<double>(d->mBasis + 2);
  d->gX = A.alloc<double>(d->N);
  d->R = A.alloc<double>(d->N);
  d->t1 = A.alloc<double>(d->N);
  d->t2 = A.alloc<double>(d->N);
  d->t3 = A.alloc<double>(d->N);
  d->xs = A.alloc<double>(d->N);
  d->rhs = A.alloc<double>(d->N);
  d->V = A.alloc<double>((size_t)(d->mBasis + 1) * d->N);
  d->Z = A.alloc<double>((size_t)d->mBasis * d->N);
  d->valT = A.alloc<double>(c->nEnt);
  CK(cudaMemsetAsync(d->dgZero, 0, sizeof(double) * 3 * c->nB, c->stream));
  CK(cudaMemsetAsync(d->zeroB, 0, sizeof(double) * c->nB, c->stream));
  // transposed momentum matrix: entry (r, c) of A^T is the stored entry (c, r) of the same face
  std::vector<int> tw(c->nEnt);
  for (int e = 0; e < c->nEnt; ++e) tw[e] = e;
  for (int f = 0; f < c->nI; ++f) {
    tw[c->slotOwn[f]] = c->slotNei[f];
    tw[c->slotNei[f]] = c->slotOwn[f];
  }
  d->twin = A.upload(tw);
  return *d;
}

AdjArgs adj_args(anb_ctx* c, AdjointData& d) {
  AdjArgs a{};
  a.U = c->U;
  a.P = c->P;
  a.G = d.G;
  a.aP = d.aP;
  a.rau = d.rau;
  a.rho = c->prm.rho;
  a.mu = c->prm.mu;
  a.uRelax = c->prm.u_relax;
  a.relax = c->prm.u_relax < 0.999999 ? 1 : 0;
  a.red = c->red;
  return a;
}

// Gradients of the state and the aP / rAU of the current (converged) state.
void base(anb_ctx* c, AdjointData& d) {
  const int C = c->C;
  const double* phi[4] = {c->U, c->U + C, c->U + 2 * C, c->P};
  const unsigned char bits[4] = {1, 2, 4, 8};
  double* out[4] = {d.G, d.G + 3 * C, d.G + 6 * C, d.G + 9 * C};
  grad(c, 4, phi, bits, out);
  adj_base(c->lc, c->dm, adj_args(c, d));
}

// dR = J dX + R_g dg + R_mu dmu (dX: 4C device, dg: 3 nB device)
void jvp(anb_ctx* c, AdjointData& d, const double* dX, const double* dg, double dmu, double* dR) {
  const int C = c->C, nB = c->nB;
  GradArgs ga{};
  ga.nf = 4;
  const unsigned char bits[4] = {1, 2, 4, 8};
  for (int q = 0; q < 4; ++q) {
    ga.phi[q] = dX + (size_t)q * C;
    ga.bit[q] = bits[q];
    ga.bval[q] = q < 3 ? dg + (size_t)q * nB : d.zeroB;
    ga.g[q] = d.dG + (size_t)3 * q * C;
  }
  launch_lsq_grad(c->lc, c->dm, ga);
  TanArgs t{};
  t.dU = dX;
  t.dp = dX + 3 * (size_t)C;
  t.dg = dg;
  t.dmu = dmu;
  t.dG = d.dG;
  t.daP = d.daP;
  adj_jvp(c->lc, c->dm, adj_args(c, d), t, dR);
}

// out = J^T w (4C); gbar (3 nB) and muBar[0] as by-products
void vjp(anb_ctx* c, AdjointData& d, const double* w, double* out) {
  AdjWork aw{};
  aw.w = w;
  aw.abar = d.abar;
  aw.h = d.h;
  aw.gbar = d.gbar;
  aw.muBar = d.muBar;
  adj_vjp(c->lc, c->dm, adj_args(c, d), aw, out);
}

// ---- preconditioner ---------------------------------------------------------------------------
// Momentum matrix at the converged state (relaxed as in the SIMPLE iteration, see AdjointData),
// its transpose, the pressure matrix from the same rAU the SIMPLE iteration uses, and its AMG
// hierarchy.
void prec_setup(anb_ctx* c, AdjointData& d) {
  MomArgs ma{};
  ma.U = c->U;
  ma.Q = c->U;
  ma.G = d.G;
  ma.rho = c->prm.rho;
  ma.mu = c->prm.mu;
  ma.uRelax = d.momRelaxed ? c->prm.u_relax : 1.0;
  ma.relax = d.momRelaxed && c->prm.u_relax < 0.999999 ? 1 : 0;
  ma.rhsOnly = 0;
  ma.val = c->mval;
  ma.diag = c->mdiag;
  ma.rhs = c->rhs;
  ma.rau = c->rau;
  launch_momentum(c->lc, c->dm, ma);
  adj_permute(c->lc, c->nEnt, d.twin, c->mval, d.valT);
  PresArgs pa{};
  pa.Us = c->U;
  pa.P = c->P;
  pa.Gp = d.G + 9 * (size_t)c->C;
  pa.rau = d.rau;
  pa.rho = c->prm.rho;
  pa.val = c->pval;
  pa.diag = c->pdiag;
  pa.phiStar = c->phiStar;
  pa.divStar = c->divStar;
  pa.b = c->pb;
  pa.pc = c->Pc;
  pa.wdinv = c->pwdinv;
  pa.omega = c->amg.omega;
  launch_pressure_rc(c->lc, c->dm, pa);
  release_amg(c);
  ensure_amg(c);
  d.precReady = true;
}


// x (3C) = M^{-1} b with M the momentum matrix (transpose when trans), from x = 0
void mom_solve(anb_ctx* c, AdjointData& d, bool trans, const double* b, double* x) {
  BicgArgs a{};
  a.A = DSell{c->C, c->dm.sliceOff, c->dm.col, trans ? d.valT : c->mval, c->mdiag, c->L.maxRowLen};
  a.nc = 3;
  a.b = b;
  a.x = x;
  a.r = c->bw[0]; a.rh = c->bw[1]; a.p = c->bw[2]; a.v = c->bw[3];
  a.s = c->bw[4]; a.t = c->bw[5]; a.ph = c->bw[6]; a.sh = c->bw[7];
  a.sc = c->scal + kScalBicg;
  a.fl = c->flags + kFlagBicg;
  a.atol = 0.0;
  a.rtol = d.momRtol;
  a.maxit = d.momMaxit;
  a.red = c->red;
  CK(cudaMemsetAsync(x, 0, sizeof(double) * 3 * c->C, c->stream));
  bicg_init(c->lc, a);
  int done = 0;
  while (true) {
    for (int k = 0; k < 8; ++k) bicg_iteration(c->lc, a);
    done += 8;
    poll(c, a.fl, 12);
    if ((c->hFlags[0] && c->hFlags[4] && c->hFlags[8]) || done > a.maxit) break;
  }
  d.momIts += std::max(c->hFlags[2], std::max(c->hFlags[6], c->hFlags[10]));
}

// x (C) = A_p^{-1} b, from x = 0 (the caller scales b)
void p_solve(anb_ctx* c, AdjointData& d, const double* b, double* x) {
  PcgArgs a = pcg_args(c, b, d.pRtol);
  a.atol = 0.0;
  a.maxit = 500;
  const AmgDev* amg = (c->prm.p_use_amg && c->amgBuilt && c->amg.nLevels >= 2) ? &c->amg : nullptr;
  CK(cudaMemsetAsync(a.x, 0, sizeof(double) * c->C, c->stream));
  pcg_init(c->lc, a);
  pcg_precondition(c->lc, a, amg);
  int it = 0;
  while (true) {
    for (int k = 0; k < 8; ++k) pcg_iteration(c->lc, a, it++, amg);
    poll(c, a.fl, 4);
    if (c->hFlags[0] || it > a.maxit) break;
  }
  CK(cudaMemcpyAsync(x, a.x, sizeof(double) * c->C, cudaMemcpyDeviceToDevice, c->stream));
  d.pIts += c->hFlags[1];
}

void scale(anb_ctx* c, AdjointData& d, size_t n, const double* src, double s, double* dst) {
  CK(cudaMemcpyAsync(d.coef, &s, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  vec_lincomb(c->lc, n, 1, src, n, d.coef, 0.0, dst);
}
// dst = a * x + b * y  (n)
void axpby(anb_ctx* c, AdjointData& d, size_t n, double a, const double* x, double b, double* y) {
  CK(cudaMemcpyAsync(d.coef, &a, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  vec_lincomb(c->lc, n, 1, x, n, d.coef, b, y);
}

// z = P^{-1} s (forward) or P^{-T} s (transposed); s, z: 4C.  Uses t1..t3 as work.
void precondition(anb_ctx* c, AdjointData& d, bool trans, const double* s, double* z) {
  const int C = c->C;
  const double rho = c->prm.rho, fac = c->prm.u_relax < 0.999999 ? 1.0 / c->prm.u_relax : 1.0;
  double* zU = z;
  double* zp = z + 3 * (size_t)C;
  if (!trans) {
    mom_solve(c, d, false, s, zU);                                  // dU* = A^-1 s_U
    adj_div_u(c->lc, c->dm, rho, zU, d.t1);                         // D_U dU*
    CK(cudaMemcpyAsync(d.t2, s + 3 * (size_t)C, sizeof(double) * C, cudaMemcpyDeviceToDevice, c->stream));
    axpby(c, d, C, -d.schur / rho, d.t1, d.schur / rho, d.t2);    // uRelax (s_c - D_U dU*) / rho
    p_solve(c, d, d.t2, zp);                                        // dp
    GradArgs ga{};
    ga.nf = 1;
    ga.phi[0] = zp;
    ga.bit[0] = 8;
    ga.bval[0] = d.zeroB;
    ga.g[0] = d.t3;
    launch_lsq_grad(c->lc, c->dm, ga);
    adj_sub_scaled_grad(c->lc, C, d.rau, fac, d.t3, zU);            // dU = dU* - (rAU/uRelax) grad dp
  } else {
    adj_grad_t(c->lc, c->dm, d.rau, fac, s, d.t3, 8u, d.t1);        // (Dinv G)^T s_U
    CK(cudaMemcpyAsync(d.t2, s + 3 * (size_t)C, sizeof(double) * C, cudaMemcpyDeviceToDevice, c->stream));
    axpby(c, d, C, -d.schur / rho, d.t1, d.schur / rho, d.t2);    // uRelax (s_c - ...) / rho
    p_solve(c, d, d.t2, zp);
    adj_div_u_t(c->lc, c->dm, rho, zp, d.t1);                       // D_U^T z_p
    CK(cudaMemcpyAsync(d.t2, s, sizeof(double) * 3 * C, cudaMemcpyDeviceToDevice, c->stream));
    axpby(c, d, 3 * (size_t)C, -1.0, d.t1, 1.0, d.t2);              // s_U - D_U^T z_p
    mom_solve(c, d, true, d.t2, zU);                                // A^-T (...)
  }
}

double norm(anb_ctx* c, AdjointData& d, size_t n, const double* x) {
  vec_mdot(c->lc, n, 1, x, n, x, d.partials, d.coef);
  double v = 0.0;
  CK(cudaMemcpyAsync(&v, d.coef, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return std::sqrt(std::max(v, 0.0));
}

// K x = b with K = J (trans = false) or J^T, right-preconditioned restarted FGMRES from x = 0.
// Stops at |b - K x| <= rtol |b|.
struct KrylovResult {
  int its = 0;
  bool conv = false;
  double res = 0.0, bnorm = 0.0;
};
KrylovResult fgmres(anb_ctx* c, AdjointData& d, bool trans, const double* b, double* x, double rtol, int maxIt) {
  const size_t N = d.N;
  const int m = d.mBasis;
  KrylovResult kr;
  CK(cudaMemsetAsync(x, 0, sizeof(double) * N, c->stream));
  kr.bnorm = norm(c, d, N, b);
  if (kr.bnorm == 0.0) {
    kr.conv = true;
    return kr;
  }
  const double target = rtol * kr.bnorm;
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), gvec(m + 1), y(m), hcol(m + 2), h2(m + 2);
  bool first = true;
  while (kr.its < maxIt) {
    // r = b - K x (the first cycle starts from x = 0)
    double* r = d.V;
    if (first) {
      CK(cudaMemcpyAsync(r, b, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
    } else {
      if (trans) vjp(c, d, x, d.t3);
      else jvp(c, d, x, d.dgZero, 0.0, d.t3);
      CK(cudaMemcpyAsync(r, b, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
      axpby(c, d, N, -1.0, d.t3, 1.0, r);
    }
    first = false;
    const double beta = norm(c, d, N, r);
    kr.res = beta;
    if (beta <= target) {
      kr.conv = true;
      break;
    }
    scale(c, d, N, r, 1.0 / beta, r);
    std::fill(gvec.begin(), gvec.end(), 0.0);
    gvec[0] = beta;
    int j = 0;
    for (; j < m && kr.its < maxIt; ++j) {
      double* vj = d.V + (size_t)j * N;
      double* zj = d.Z + (size_t)j * N;
      double* w = d.V + (size_t)(j + 1) * N;
      precondition(c, d, trans, vj, zj);
      if (trans) vjp(c, d, zj, w);
      else jvp(c, d, zj, d.dgZero, 0.0, w);
      ++kr.its;
      // classical Gram-Schmidt, twice
      for (int pass = 0; pass < 2; ++pass) {
        vec_mdot(c->lc, N, j + 1, d.V, N, w, d.partials, d.coef);
        CK(cudaMemcpyAsync(h2.data(), d.coef, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int i = 0; i <= j; ++i) {
          hcol[i] = (pass ? hcol[i] : 0.0) + h2[i];
          h2[i] = -h2[i];
        }
        CK(cudaMemcpyAsync(d.coef, h2.data(), sizeof(double) * (j + 1), cudaMemcpyHostToDevice, c->stream));
        vec_lincomb(c->lc, N, j + 1, d.V, N, d.coef, 1.0, w);
      }
      const double hn = norm(c, d, N, w);
      hcol[j + 1] = hn;
      if (hn > 0.0) scale(c, d, N, w, 1.0 / hn, w);
      // Givens rotations
      for (int i = 0; i < j; ++i) {
        const double t = cs[i] * hcol[i] + sn[i] * hcol[i + 1];
        hcol[i + 1] = -sn[i] * hcol[i] + cs[i] * hcol[i + 1];
        hcol[i] = t;
      }
      const double den = std::hypot(hcol[j], hcol[j + 1]);
      cs[j] = den > 0.0 ? hcol[j] / den : 1.0;
      sn[j] = den > 0.0 ? hcol[j + 1] / den : 0.0;
      hcol[j] = den;
      hcol[j + 1] = 0.0;
      gvec[j + 1] = -sn[j] * gvec[j];
      gvec[j] = cs[j] * gvec[j];
      for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = hcol[i];
      kr.res = std::fabs(gvec[j + 1]);
      if (kr.res <= target || hn == 0.0) {
        ++j;
        break;
      }
    }
    // x += Z y, H y = g (upper triangular j x j)
    for (int i = j - 1; i >= 0; --i) {
      double s = gvec[i];
      for (int k = i + 1; k < j; ++k) s -= H[(size_t)i * m + k] * y[k];
      y[i] = H[(size_t)i * m + i] != 0.0 ? s / H[(size_t)i * m + i] : 0.0;
    }
    CK(cudaMemcpyAsync(d.coef, y.data(), sizeof(double) * j, cudaMemcpyHostToDevice, c->stream));
    vec_lincomb(c->lc, N, j, d.Z, N, d.coef, 1.0, x);
    if (kr.res <= target) {
      // confirm with the true residual
      if (trans) vjp(c, d, x, d.t3);
      else jvp(c, d, x, d.dgZero, 0.0, d.t3);
      CK(cudaMemcpyAsync(d.t2, b, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
      axpby(c, d, N, -1.0, d.t3, 1.0, d.t2);
      kr.res = norm(c, d, N, d.t2);
      if (kr.res <= 1.5 * target) {
        kr.conv = true;
        break;
      }
    }
  }
  return kr;
}

ObjArgs obj_args(anb_ctx* c, AdjointData& d, int patch, int sign, const double dir[3]) {
  if (patch < 0 || patch >= (int)c->hm.patches.size()) throw AnbError(ANB_ERR_INVALID, "invalid patch index");
  ObjArgs o{};
  o.b0 = c->hm.patches[patch].start - c->nI;
  o.b1 = o.b0 + c->hm.patches[patch].nFaces;
  o.sign = sign;
  for (int k = 0; k < 3; ++k) o.dir[k] = dir[k];
  o.bA = c->dBA;
  o.bN = c->dBN;
  o.val = d.objVal;
  return o;
}

void fill_info(anb_adjoint_info* info, const KrylovResult& kr, double secs, const AdjointData* d = nullptr) {
  if (!info) return;
  if (d) {
    info->prec_mom_its = (int)d->momIts;
    info->prec_p_its = (int)d->pIts;
  }
  info->iterations = kr.its;
  info->converged = kr.conv ? 1 : 0;
  info->res_norm = kr.res;
  info->rhs_norm = kr.bnorm;
  info->seconds = secs;
}

void upload4(anb_ctx* c, const double* src, double* dst) {
  const size_t C = c->C;
  const double* s4[4] = {src, src + C, src + 2 * C, src + 3 * C};
  upload_cells(c, s4, dst, 4);
}
void download4(anb_ctx* c, const double* src, double* dst) {
  const size_t C = c->C;
  double* d4[4] = {dst, dst + C, dst + 2 * C, dst + 3 * C};
  download_cells(c, src, d4, 4);
}
// Dirichlet-value arrays: 3 x nFaces (input order) <-> 3 x nBoundary (device)
void upload_bc3(anb_ctx* c, const double* src, double* dst) {
  std::vector<double> h((size_t)3 * c->nB, 0.0);
  if (src)
    for (int q = 0; q < 3; ++q)
      for (int b = 0; b < c->nB; ++b) h[(size_t)q * c->nB + b] = src[(size_t)q * (c->nI + c->nB) + c->nI + b];
  CK(cudaMemcpyAsync(dst, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}
void download_bc3(anb_ctx* c, const double* src, double* dst) {
  std::vector<double> h((size_t)3 * c->nB);
  CK(cudaMemcpyAsync(h.data(), src, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const size_t F = (size_t)c->nI + c->nB;
  std::vector<uint8_t> ty(c->nB);
  CK(cudaMemcpy(ty.data(), c->dBType, c->nB, cudaMemcpyDeviceToHost));
  for (int q = 0; q < 3; ++q) {
    for (int f = 0; f < c->nI; ++f) dst[q * F + f] = 0.0;
    for (int b = 0; b < c->nB; ++b)  // only Dirichlet values are parameters
      dst[q * F + c->nI + b] = (ty[b] & (1u << q)) ? h[(size_t)q * c->nB + b] : 0.0;
  }
}

void require(anb_ctx* c) {
  check_ready(c);
  if (c->mixed) throw AnbError(ANB_ERR_UNSUPPORTED, "this entry point needs an FP64 (ANB_PRECISION_FP64) context");
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace
}  // namespace anb

using namespace anb;

extern "C" {

int anb_set_viscosity(anb_ctx* c, double mu) {
  if (!c || !(mu > 0.0)) return ANB_ERR_INVALID;
  c->prm.mu = mu;
  return ANB_OK;
}

int anb_steady_residual(anb_ctx* c, double* res, double* norms) {
  if (!c) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    require(c);
    AdjointData& d = adj(c);
    base(c, d);
    adj_residual(c->lc, c->dm, adj_args(c, d), d.R);
    if (norms) {
      norms[0] = norm(c, d, 3 * (size_t)c->C, d.R);
      norms[1] = norm(c, d, (size_t)c->C, d.R + 3 * (size_t)c->C);
    }
    if (res) download4(c, d.R, res);
    CK(cudaStreamSynchronize(c->stream));
    return ANB_OK;
  });
}

int anb_force_objective(anb_ctx* c, int patch, int sign, const double dir[3], double* J, double* dJ_dmu_explicit) {
  if (!c || !dir || !J) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    require(c);
    AdjointData& d = adj(c);
    base(c, d);
    adj_objective(c->lc, c->dm, adj_args(c, d), obj_args(c, d, patch, sign, dir), d.gX);
    double v[2];
    CK(cudaMemcpyAsync(v, d.objVal, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *J = v[0];
    if (dJ_dmu_explicit) *dJ_dmu_explicit = v[1];
    return ANB_OK;
  });
}

int anb_debug_jvp(anb_ctx* c, const double* dX, const double* dbc, double dmu, double* dR) {
  if (!c || !dX || !dR) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    require(c);
    AdjointData& d = adj(c);
    base(c, d);
    upload4(c, dX, d.t1);
    upload_bc3(c, dbc, d.dgDir);
    jvp(c, d, d.t1, d.dgDir, dmu, d.t2);
    download4(c, d.t2, dR);
    return ANB_OK;
  });
}

int anb_debug_vjp(anb_ctx* c, const double* w, double* out, double* gbc, double* gmu) {
  if (!c || !w || !out) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    require(c);
    AdjointData& d = adj(c);
    base(c, d);
    upload4(c, w, d.t1);
    vjp(c, d, d.t1, d.t2);
    download4(c, d.t2, out);
    if (gbc) download_bc3(c, d.gbar, gbc);
    if (gmu) CK(cudaMemcpy(gmu, d.muBar, sizeof(double), cudaMemcpyDeviceToHost));
    return ANB_OK;
  });
}

int anb_newton_solve(anb_ctx* c, int maxNewton, double tol, int linMaxIt, int* steps, double* resNorm,
                     anb_adjoint_info* info) {
  if (!c) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    require(c);
    const auto t0 = std::chrono::steady_clock::now();
    AdjointData& d = adj(c);
    d.momIts = d.pIts = 0;
    KrylovResult kr{};
    int k = 0, total = 0;
    double rn = 0.0;
    for (;; ++k) {
      base(c, d);
      adj_residual(c->lc, c->dm, adj_args(c, d), d.R);
      rn = norm(c, d, d.N, d.R);
      if (rn <= tol || k >= maxNewton) break;
      prec_setup(c, d);
      scale(c, d, d.N, d.R, -1.0, d.rhs);
      kr = fgmres(c, d, false, d.rhs, d.xs, 1e-3, linMaxIt);
      total += kr.its;
      // X += dX
      axpby(c, d, 3 * (size_t)c->C, 1.0, d.xs, 1.0, c->U);
      axpby(c, d, (size_t)c->C, 1.0, d.xs + 3 * (size_t)c->C, 1.0, c->P);
    }
    if (steps) *steps = k;
    if (resNorm) *resNorm = rn;
    kr.its = total;
    kr.res = rn;
    fill_info(info, kr, seconds_since(t0), &d);
    if (info) info->converged = rn <= tol ? 1 : 0;
    return rn <= tol ? ANB_OK : ANB_NOT_CONVERGED;
  });
}

int anb_tangent_linear(anb_ctx* c, int patch, int sign, const double dir[3], const double* dbc, double dmu,
                       double* dJ, anb_adjoint_info* info) {
  if (!c || !dir || !dJ) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    require(c);
    const auto t0 = std::chrono::steady_clock::now();
    AdjointData& d = adj(c);
    d.momIts = d.pIts = 0;
    base(c, d);
    prec_setup(c, d);
    upload_bc3(c, dbc, d.dgDir);
    CK(cudaMemsetAsync(d.t1, 0, sizeof(double) * d.N, c->stream));
    jvp(c, d, d.t1, d.dgDir, dmu, d.rhs);  // R_theta dtheta
    scale(c, d, d.N, d.rhs, -1.0, d.rhs);
    KrylovResult kr = fgmres(c, d, false, d.rhs, d.xs, d.rtol, 2000);
    adj_objective(c->lc, c->dm, adj_args(c, d), obj_args(c, d, patch, sign, dir), d.gX);
    vec_mdot(c->lc, d.N, 1, d.gX, d.N, d.xs, d.partials, d.coef);
    double v[2], jx = 0.0;
    CK(cudaMemcpyAsync(&jx, d.coef, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(v, d.objVal, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *dJ = jx + v[1] * dmu;
    fill_info(info, kr, seconds_since(t0), &d);
    return kr.conv ? ANB_OK : ANB_NOT_CONVERGED;
  });
}

int anb_adjoint_force_grad(anb_ctx* c, int patch, int sign, const double dir[3], double* dJ_dbc, double* dJ_dmu,
                           double* J, anb_adjoint_info* info) {
  if (!c || !dir) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    require(c);
    const auto t0 = std::chrono::steady_clock::now();
    AdjointData& d = adj(c);
    d.momIts = d.pIts = 0;
    base(c, d);
    prec_setup(c, d);
    adj_objective(c->lc, c->dm, adj_args(c, d), obj_args(c, d, patch, sign, dir), d.gX);
    KrylovResult kr = fgmres(c, d, true, d.gX, d.xs, d.rtol, 2000);  // J^T lambda = dJ/dX
    vjp(c, d, d.xs, d.t1);                                           // gbar = R_g^T lambda, muBar
    double v[2], mb = 0.0;
    CK(cudaMemcpyAsync(v, d.objVal, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&mb, d.muBar, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (J) *J = v[0];
    if (dJ_dmu) *dJ_dmu = v[1] - mb;
    if (dJ_dbc) {
      download_bc3(c, d.gbar, dJ_dbc);
      const size_t n = (size_t)3 * (c->nI + c->nB);
      for (size_t i = 0; i < n; ++i) dJ_dbc[i] = -dJ_dbc[i];
    }
    fill_info(info, kr, seconds_since(t0), &d);
    return kr.conv ? ANB_OK : ANB_NOT_CONVERGED;
  });
}

}  // extern "C"
