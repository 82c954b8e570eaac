// CPU oracle: restatement of the reference's SIMPLE outer iteration (generic_simple_v1).
// TEST INFRASTRUCTURE ONLY - see oracle.h.  "GSV1" = apps/generic_simple_v1/src/main.cu.
#include "oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using V3 = std::array<double, 3>;
inline V3 add3(const V3& a, const V3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline V3 sub3(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline V3 mul3(double s, const V3& a) { return {s * a[0], s * a[1], s * a[2]}; }
inline double dot3(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline V3 cross3(const V3& a, const V3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline double norm3(const V3& a) { return std::sqrt(dot3(a, a)); }

// Deterministic parallel sum: fixed 4096-element chunks, partials added in chunk order.
template <class F>
double det_sum(int n, F f) {
  const int CH = 4096;
  int nch = (n + CH - 1) / CH;
  std::vector<double> part(std::max(nch, 1), 0.0);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nch; ++k) {
    double s = 0.0;
    int e = std::min(n, (k + 1) * CH);
    for (int i = k * CH; i < e; ++i) s += f(i);
    part[k] = s;
  }
  double s = 0.0;
  for (double v : part) s += v;
  return s;
}

struct CSR {  // reference MatrixPattern (GSV1:1011-1020, 1315-1374), diagonal included
  int n = 0;
  std::vector<int> rowOff, cols, diagPos, fPP, fPN, fNP, fNN;
  std::vector<double> vals;
};

}  // namespace

struct orc_mesh {
  // topology (GSV1 Mesh, main.cu:61-72)
  std::vector<V3> P;
  std::vector<std::vector<int>> faces;
  std::vector<int> owner, neigh, bPatch, patchStart, patchN;
  int nFaces = 0, nInternal = 0, nCells = 0;
  std::vector<V3> cc, xf, nf, Sf;
  std::vector<double> vol, Af;
  std::vector<std::vector<int>> cellNbrs, cellBFace, cellFaces, cellOrient;
  double maxNonOrthDeg = 0.0;
  // LSQ operator (build_lsq_gradient_operator, GSV1:1159-1251)
  std::vector<int> gOff, gSrc, gFace;
  std::vector<double> gcx, gcy, gcz;
  CSR pat;
  // BC (DeviceBC, GSV1:1003-1009): per patch type and per face value for u, v, w, p
  std::vector<int> type[4];
  std::vector<double> fval[4];
};

namespace {

// read_openfoam_polymesh geometry part, GSV1:584-597 (same operation order).
void build_geometry(orc_mesh& m) {
  m.nCells = 0;
  for (int v : m.owner) m.nCells = std::max(m.nCells, v + 1);
  for (int v : m.neigh) m.nCells = std::max(m.nCells, v + 1);
  m.cellFaces.assign(m.nCells, {});
  m.cellOrient.assign(m.nCells, {});
  for (int f = 0; f < m.nFaces; ++f) {
    m.cellFaces[m.owner[f]].push_back(f);
    m.cellOrient[m.owner[f]].push_back(+1);
  }
  for (int f = 0; f < m.nInternal; ++f) {
    m.cellFaces[m.neigh[f]].push_back(f);
    m.cellOrient[m.neigh[f]].push_back(-1);
  }
  m.cc.assign(m.nCells, {0, 0, 0});
  m.vol.assign(m.nCells, 0.0);
  std::string bad;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < m.nCells; ++c) {
    std::set<int> vs;
    for (int f : m.cellFaces[c])
      for (int v : m.faces[f]) vs.insert(v);
    V3 c0{0, 0, 0};
    for (int v : vs) c0 = add3(c0, m.P[v]);
    c0 = mul3(1.0 / std::max((int)vs.size(), 1), c0);
    double Vc = 0.0;
    V3 M{0, 0, 0};
    for (size_t j = 0; j < m.cellFaces[c].size(); ++j) {
      std::vector<int> fv = m.faces[m.cellFaces[c][j]];
      if (m.cellOrient[c][j] < 0) std::reverse(fv.begin(), fv.end());
      V3 a = m.P[fv[0]];
      for (size_t i = 1; i + 1 < fv.size(); ++i) {
        V3 b = m.P[fv[i]], d = m.P[fv[i + 1]];
        double vT = dot3(sub3(a, c0), cross3(sub3(b, c0), sub3(d, c0))) / 6.0;
        V3 cT = mul3(0.25, add3(add3(c0, a), add3(b, d)));
        Vc += vT;
        M = add3(M, mul3(vT, cT));
      }
    }
    if (Vc <= 0) {
#pragma omp critical
      bad = "Non-positive cell volume at cell " + std::to_string(c);
    } else {
      m.vol[c] = Vc;
      m.cc[c] = mul3(1.0 / Vc, M);
    }
  }
  if (!bad.empty()) throw std::runtime_error(bad);
  m.xf.assign(m.nFaces, {0, 0, 0});
  m.Af.assign(m.nFaces, 0.0);
  m.nf.assign(m.nFaces, {0, 0, 0});
  m.Sf.assign(m.nFaces, {0, 0, 0});
  for (int f = 0; f < m.nFaces; ++f) {
    V3 x{0, 0, 0};
    for (int v : m.faces[f]) x = add3(x, m.P[v]);
    x = mul3(1.0 / std::max((int)m.faces[f].size(), 1), x);
    m.xf[f] = x;
    V3 a = m.P[m.faces[f][0]];
    V3 av{0, 0, 0};
    for (size_t i = 1; i + 1 < m.faces[f].size(); ++i) {
      V3 b = m.P[m.faces[f][i]], d = m.P[m.faces[f][i + 1]];
      av = add3(av, mul3(0.5, cross3(sub3(b, a), sub3(d, a))));
    }
    double am = norm3(av);
    if (am <= 1e-30) throw std::runtime_error("Degenerate face area at face " + std::to_string(f));
    V3 nl = mul3(1.0 / am, av);
    int Pc = m.owner[f];
    V3 dt = (f < m.nInternal) ? sub3(m.cc[m.neigh[f]], m.cc[Pc]) : sub3(m.xf[f], m.cc[Pc]);
    if (dot3(nl, dt) < 0) nl = mul3(-1.0, nl);
    m.Af[f] = am;
    m.nf[f] = nl;
    m.Sf[f] = mul3(am, nl);
  }
  m.cellNbrs.assign(m.nCells, {});
  m.cellBFace.assign(m.nCells, {});
  for (int f = 0; f < m.nFaces; ++f) {
    int Pc = m.owner[f];
    if (f < m.nInternal) {
      m.cellNbrs[Pc].push_back(m.neigh[f]);
      m.cellNbrs[m.neigh[f]].push_back(Pc);
    } else {
      m.cellBFace[Pc].push_back(f);
    }
  }
  for (auto& nb : m.cellNbrs) {
    std::sort(nb.begin(), nb.end());
    nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
  }
  m.maxNonOrthDeg = 0.0;
  for (int f = 0; f < m.nInternal; ++f) {
    V3 d = sub3(m.cc[m.neigh[f]], m.cc[m.owner[f]]);
    double ca = std::fabs(dot3(d, m.nf[f])) / std::max(norm3(d), 1e-30);
    ca = std::min(1.0, std::max(0.0, ca));
    m.maxNonOrthDeg = std::max(m.maxNonOrthDeg, std::acos(ca) * 180.0 / M_PI);
  }
}

// build_lsq_gradient_operator, GSV1:1159-1251.
void build_lsq(orc_mesh& m) {
  m.gOff.assign(m.nCells + 1, 0);
  m.gSrc.clear(); m.gFace.clear(); m.gcx.clear(); m.gcy.clear(); m.gcz.clear();
  for (int Pc = 0; Pc < m.nCells; ++Pc) {
    V3 xP = m.cc[Pc];
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    struct Term { int src, face; double r[3], w; };
    std::vector<Term> terms;
    for (int N : m.cellNbrs[Pc]) {
      V3 r = sub3(m.cc[N], xP);
      double w = 1.0 / std::max(dot3(r, r), 1e-30);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i][j] += w * r[i] * r[j];
      terms.push_back({N, -1, {r[0], r[1], r[2]}, w});
    }
    for (int f : m.cellBFace[Pc]) {
      V3 r = sub3(m.xf[f], xP);
      double w = 1.0 / std::max(dot3(r, r), 1e-30);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i][j] += w * r[i] * r[j];
      terms.push_back({-1, f, {r[0], r[1], r[2]}, w});
    }
    double a = M[0][0], b = M[0][1], c = M[0][2], d = M[1][0], e = M[1][1], f2 = M[1][2], g = M[2][0],
           h = M[2][1], k = M[2][2];
    double det = a * (e * k - f2 * h) - b * (d * k - f2 * g) + c * (d * h - e * g);
    double inv[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (std::fabs(det) > 1e-20) {
      inv[0][0] = (e * k - f2 * h) / det; inv[0][1] = (c * h - b * k) / det; inv[0][2] = (b * f2 - c * e) / det;
      inv[1][0] = (f2 * g - d * k) / det; inv[1][1] = (a * k - c * g) / det; inv[1][2] = (c * d - a * f2) / det;
      inv[2][0] = (d * h - e * g) / det; inv[2][1] = (b * g - a * h) / det; inv[2][2] = (a * e - b * d) / det;
    }
    m.gOff[Pc] = (int)m.gSrc.size();
    for (const auto& t : terms) {
      double bx = t.w * t.r[0], by = t.w * t.r[1], bz = t.w * t.r[2];
      m.gSrc.push_back(t.src);
      m.gFace.push_back(t.face);
      m.gcx.push_back(inv[0][0] * bx + inv[0][1] * by + inv[0][2] * bz);
      m.gcy.push_back(inv[1][0] * bx + inv[1][1] * by + inv[1][2] * bz);
      m.gcz.push_back(inv[2][0] * bx + inv[2][1] * by + inv[2][2] * bz);
    }
  }
  m.gOff[m.nCells] = (int)m.gSrc.size();
}

// build_momentum_pattern / build_pressure_pattern without anchor, GSV1:1315-1374.
void build_pattern(orc_mesh& m) {
  CSR& p = m.pat;
  p.n = m.nCells;
  p.rowOff.assign(m.nCells + 1, 0);
  p.diagPos.assign(m.nCells, 0);
  std::vector<std::map<int, int>> pos(m.nCells);
  for (int c = 0; c < m.nCells; ++c) {
    std::vector<int> cols = m.cellNbrs[c];
    cols.insert(cols.begin(), c);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    p.rowOff[c + 1] = p.rowOff[c] + (int)cols.size();
    for (size_t j = 0; j < cols.size(); ++j) pos[c][cols[j]] = p.rowOff[c] + (int)j;
  }
  p.cols.assign(p.rowOff.back(), 0);
  for (int c = 0; c < m.nCells; ++c) {
    for (auto& kv : pos[c]) p.cols[kv.second] = kv.first;
    p.diagPos[c] = pos[c][c];
  }
  p.fPP.resize(m.nInternal); p.fPN.resize(m.nInternal); p.fNP.resize(m.nInternal); p.fNN.resize(m.nInternal);
  for (int f = 0; f < m.nInternal; ++f) {
    int Pc = m.owner[f], N = m.neigh[f];
    p.fPP[f] = pos[Pc][Pc]; p.fPN[f] = pos[Pc][N]; p.fNP[f] = pos[N][Pc]; p.fNN[f] = pos[N][N];
  }
  p.vals.assign(p.rowOff.back(), 0.0);
}

// kernel_apply_lsq_gradient, GSV1:1403-1440.
void lsq_grad(const orc_mesh& m, int field, const double* phi, double* gx, double* gy, double* gz) {
  const auto& tp = m.type[field];
  const auto& fv = m.fval[field];
#pragma omp parallel for schedule(static)
  for (int Pc = 0; Pc < m.nCells; ++Pc) {
    double phiP = phi[Pc], sx = 0, sy = 0, sz = 0;
    for (int t = m.gOff[Pc]; t < m.gOff[Pc + 1]; ++t) {
      double val = phiP;
      int s = m.gSrc[t];
      if (s >= 0) val = phi[s];
      else {
        int f = m.gFace[t];
        int patch = m.bPatch[f] - 1;
        if (patch >= 0 && tp[patch] == 1) val = fv[f];
      }
      double dphi = val - phiP;
      sx += m.gcx[t] * dphi;
      sy += m.gcy[t] * dphi;
      sz += m.gcz[t] * dphi;
    }
    gx[Pc] = sx; gy[Pc] = sy; gz[Pc] = sz;
  }
}

struct G3 { std::vector<double> x, y, z; explicit G3(int n) : x(n), y(n), z(n) {} };

inline double lam_of(const orc_mesh& m, int f, const V3& d) {
  double den = dot3(d, d);
  double lam = dot3(sub3(m.xf[f], m.cc[m.owner[f]]), d) / (den > 1e-30 ? den : 1e-30);
  return std::min(1.0, std::max(0.0, lam));
}

// assemble_momentum_on_gpu_device_grad (K25, K4, K2, K3), GSV1:2346-2427, 1678-1684, 1804-1896.
void mom_full(orc_mesh& m, double rho, double mu, const double* qOld, int field, const G3& gQ,
              const double* gradPcomp, const double* uC, const double* vC, const double* wC, std::vector<double>& rhs) {
  CSR& p = m.pat;
  std::fill(p.vals.begin(), p.vals.end(), 0.0);
  (void)qOld;
  for (int c = 0; c < m.nCells; ++c) {
    p.vals[p.diagPos[c]] = 0.0;
    rhs[c] = -gradPcomp[c] * m.vol[c];
  }
  const double corrPsi = 1.0;
  for (int f = 0; f < m.nInternal; ++f) {
    int Pc = m.owner[f], N = m.neigh[f];
    V3 d = sub3(m.cc[N], m.cc[Pc]);
    double nd = dot3(m.nf[f], d);
    if (nd <= 1e-14) continue;
    double af = m.Af[f], alpha = mu * af / nd;
    double tx = mu * (m.Sf[f][0] - (af / nd) * d[0]), ty = mu * (m.Sf[f][1] - (af / nd) * d[1]),
           tz = mu * (m.Sf[f][2] - (af / nd) * d[2]);
    double lam = lam_of(m, f, d);
    double gfx = (1.0 - lam) * gQ.x[Pc] + lam * gQ.x[N], gfy = (1.0 - lam) * gQ.y[Pc] + lam * gQ.y[N],
           gfz = (1.0 - lam) * gQ.z[Pc] + lam * gQ.z[N];
    double corr = corrPsi * (gfx * tx + gfy * ty + gfz * tz);
    double ucf = (1.0 - lam) * uC[Pc] + lam * uC[N], vcf = (1.0 - lam) * vC[Pc] + lam * vC[N],
           wcf = (1.0 - lam) * wC[Pc] + lam * wC[N];
    double F = rho * af * (ucf * m.nf[f][0] + vcf * m.nf[f][1] + wcf * m.nf[f][2]);
    p.vals[p.fPP[f]] += alpha + F * (1.0 - lam);
    p.vals[p.fPN[f]] += -alpha + F * lam;
    p.vals[p.fNP[f]] += -alpha - F * (1.0 - lam);
    p.vals[p.fNN[f]] += alpha - F * lam;
    rhs[Pc] += corr;
    rhs[N] += -corr;
  }
  for (int f = m.nInternal; f < m.nFaces; ++f) {
    int Pc = m.owner[f], patch = m.bPatch[f] - 1;
    V3 d = sub3(m.xf[f], m.cc[Pc]);
    double nd = dot3(m.nf[f], d);
    if (nd <= 1e-14) continue;
    double af = m.Af[f], alpha = mu * af / nd;
    double tx = mu * (m.Sf[f][0] - (af / nd) * d[0]), ty = mu * (m.Sf[f][1] - (af / nd) * d[1]),
           tz = mu * (m.Sf[f][2] - (af / nd) * d[2]);
    int dg = p.diagPos[Pc];
    bool qDir = m.type[field][patch] == 1;
    if (qDir) {
      double g = m.fval[field][f];
      double corr = corrPsi * (gQ.x[Pc] * tx + gQ.y[Pc] * ty + gQ.z[Pc] * tz);
      p.vals[dg] += alpha;
      rhs[Pc] += alpha * g + corr;
    }
    double ucb = m.type[0][patch] == 1 ? m.fval[0][f] : uC[Pc];
    double vcb = m.type[1][patch] == 1 ? m.fval[1][f] : vC[Pc];
    double wcb = m.type[2][patch] == 1 ? m.fval[2][f] : wC[Pc];
    double F = rho * af * (ucb * m.nf[f][0] + vcb * m.nf[f][1] + wcb * m.nf[f][2]);
    if (qDir) rhs[Pc] += -F * m.fval[field][f];
    else p.vals[dg] += F;
  }
}

// assemble_momentum_rhs_only_on_gpu_device_grad (K26, K9, K7, K8, K10), GSV1:2429-2510.
void mom_rhs_only(const orc_mesh& m, double rho, double mu, double uRelax, const double* qOld, int field,
                  const G3& gQ, const double* gradPcomp, const double* uC, const double* vC, const double* wC,
                  std::vector<double>& rhs) {
  const CSR& p = m.pat;
  for (int c = 0; c < m.nCells; ++c) rhs[c] = -gradPcomp[c] * m.vol[c];
  const double corrPsi = 1.0;
  for (int f = 0; f < m.nInternal; ++f) {
    int Pc = m.owner[f], N = m.neigh[f];
    V3 d = sub3(m.cc[N], m.cc[Pc]);
    double nd = dot3(m.nf[f], d);
    if (nd <= 1e-14) continue;
    double af = m.Af[f];
    double tx = mu * (m.Sf[f][0] - (af / nd) * d[0]), ty = mu * (m.Sf[f][1] - (af / nd) * d[1]),
           tz = mu * (m.Sf[f][2] - (af / nd) * d[2]);
    double lam = lam_of(m, f, d);
    double gfx = (1.0 - lam) * gQ.x[Pc] + lam * gQ.x[N], gfy = (1.0 - lam) * gQ.y[Pc] + lam * gQ.y[N],
           gfz = (1.0 - lam) * gQ.z[Pc] + lam * gQ.z[N];
    double corr = corrPsi * (gfx * tx + gfy * ty + gfz * tz);
    rhs[Pc] += corr;
    rhs[N] += -corr;
  }
  for (int f = m.nInternal; f < m.nFaces; ++f) {
    int Pc = m.owner[f], patch = m.bPatch[f] - 1;
    V3 d = sub3(m.xf[f], m.cc[Pc]);
    double nd = dot3(m.nf[f], d);
    if (nd <= 1e-14) continue;
    double af = m.Af[f], alpha = mu * af / nd;
    double tx = mu * (m.Sf[f][0] - (af / nd) * d[0]), ty = mu * (m.Sf[f][1] - (af / nd) * d[1]),
           tz = mu * (m.Sf[f][2] - (af / nd) * d[2]);
    bool qDir = m.type[field][patch] == 1;
    if (qDir) {
      double g = m.fval[field][f];
      double corr = corrPsi * (gQ.x[Pc] * tx + gQ.y[Pc] * ty + gQ.z[Pc] * tz);
      rhs[Pc] += alpha * g + corr;
    }
    double ucb = m.type[0][patch] == 1 ? m.fval[0][f] : uC[Pc];
    double vcb = m.type[1][patch] == 1 ? m.fval[1][f] : vC[Pc];
    double wcb = m.type[2][patch] == 1 ? m.fval[2][f] : wC[Pc];
    double F = rho * af * (ucb * m.nf[f][0] + vcb * m.nf[f][1] + wcb * m.nf[f][2]);
    if (qDir) rhs[Pc] += -F * m.fval[field][f];
  }
  if (uRelax < 0.999999) {  // K10, GSV1:1787-1794
    for (int c = 0; c < m.nCells; ++c) {
      double aPold = p.vals[p.diagPos[c]] * uRelax;
      double invR = 1.0 / uRelax;
      rhs[c] += (invR - 1.0) * aPold * qOld[c];
    }
  }
}

// kernel_relax_momentum_system (GSV1:1686-1695) and kernel_extract_vol_over_diag (1796-1802).
void mom_relax(orc_mesh& m, double uRelax, const double* qOld, std::vector<double>& rhs) {
  if (uRelax >= 0.999999) return;
  CSR& p = m.pat;
  for (int c = 0; c < m.nCells; ++c) {
    int dg = p.diagPos[c];
    double aP = p.vals[dg], invR = 1.0 / uRelax;
    p.vals[dg] = aP * invR;
    rhs[c] += (invR - 1.0) * aP * qOld[c];
  }
}
void extract_rau(const orc_mesh& m, std::vector<double>& rau) {
  for (int c = 0; c < m.nCells; ++c) {
    double a = m.pat.vals[m.pat.diagPos[c]];
    rau[c] = std::fabs(a) > 1e-30 ? m.vol[c] / a : 0.0;
  }
}

// update_pressure_matrix_from_rAU (K25, K11, K12), GSV1:2532-2551, 1898-1950.
void pressure_matrix(const orc_mesh& m, const double* rau, std::vector<double>& vals) {
  const CSR& p = m.pat;
  std::fill(vals.begin(), vals.end(), 0.0);
  for (int f = 0; f < m.nInternal; ++f) {
    int Pc = m.owner[f], N = m.neigh[f];
    V3 d = sub3(m.cc[N], m.cc[Pc]);
    double dpn = dot3(m.nf[f], d);
    if (dpn <= 1e-14) continue;
    double lam = lam_of(m, f, d);
    double rAUf = (1.0 - lam) * rau[Pc] + lam * rau[N];
    double coeff = m.Af[f] * rAUf / dpn;
    vals[p.fPP[f]] += coeff;
    vals[p.fPN[f]] += -coeff;
    vals[p.fNP[f]] += -coeff;
    vals[p.fNN[f]] += coeff;
  }
  for (int f = m.nInternal; f < m.nFaces; ++f) {
    int patch = m.bPatch[f] - 1;
    if (m.type[3][patch] != 1) continue;
    int Pc = m.owner[f];
    V3 d = sub3(m.xf[f], m.cc[Pc]);
    double dpn = dot3(m.nf[f], d);
    if (dpn <= 1e-14) continue;
    vals[p.diagPos[Pc]] += m.Af[f] * rau[Pc] / dpn;
  }
}

// kernel_build_rhiechow_predicted_flux_stokes_3d, GSV1:1474-1521.
void rhie_chow(const orc_mesh& m, double rho, const double* u, const double* v, const double* w, const double* p,
               const G3& gp, const double* rau, std::vector<double>& phiStar) {
#pragma omp parallel for schedule(static)
  for (int f = 0; f < m.nFaces; ++f) {
    int Pc = m.owner[f];
    if (f < m.nInternal) {
      int N = m.neigh[f];
      V3 d = sub3(m.cc[N], m.cc[Pc]);
      double dpn = dot3(m.nf[f], d);
      double den = std::max(dot3(d, d), 1.0e-30);
      double lam = dot3(sub3(m.xf[f], m.cc[Pc]), d) / den;
      lam = std::min(1.0, std::max(0.0, lam));
      double ub = (1.0 - lam) * u[Pc] + lam * u[N], vb = (1.0 - lam) * v[Pc] + lam * v[N],
             wb = (1.0 - lam) * w[Pc] + lam * w[N];
      double gx = (1.0 - lam) * gp.x[Pc] + lam * gp.x[N], gy = (1.0 - lam) * gp.y[Pc] + lam * gp.y[N],
             gz = (1.0 - lam) * gp.z[Pc] + lam * gp.z[N];
      double rAUf = (1.0 - lam) * rau[Pc] + lam * rau[N];
      double phiI = rho * m.Af[f] * (ub * m.nf[f][0] + vb * m.nf[f][1] + wb * m.nf[f][2]);
      double rc = rho * m.Af[f] * rAUf / std::max(std::fabs(dpn), 1.0e-30) *
                  ((p[N] - p[Pc]) - (gx * d[0] + gy * d[1] + gz * d[2]));
      phiStar[f] = phiI - rc;
    } else {
      int patch = m.bPatch[f] - 1;
      double uf = m.type[0][patch] == 1 ? m.fval[0][f] : u[Pc];
      double vf = m.type[1][patch] == 1 ? m.fval[1][f] : v[Pc];
      double wf = m.type[2][patch] == 1 ? m.fval[2][f] : w[Pc];
      phiStar[f] = rho * m.Af[f] * (uf * m.nf[f][0] + vf * m.nf[f][1] + wf * m.nf[f][2]);
    }
  }
}

// continuity_residual_gpu (K24 + K15), GSV1:1281-1288, 1523-1536.
void continuity(const orc_mesh& m, const std::vector<double>& phi, std::vector<double>& div) {
  std::fill(div.begin(), div.end(), 0.0);
  for (int f = 0; f < m.nFaces; ++f) {
    div[m.owner[f]] += phi[f];
    if (f < m.nInternal) div[m.neigh[f]] -= phi[f];
  }
}

// kernel_pressure_nonorth_flux_and_divergence, GSV1:1538-1593.
void nonorth(const orc_mesh& m, const double* rau, const G3& g, std::vector<double>& phiNO,
             std::vector<double>& divNO) {
  std::fill(divNO.begin(), divNO.end(), 0.0);
  for (int f = 0; f < m.nFaces; ++f) {
    double flux = 0.0;
    if (f < m.nInternal) {
      int Pc = m.owner[f], N = m.neigh[f];
      V3 d = sub3(m.cc[N], m.cc[Pc]);
      double dpn = dot3(m.nf[f], d);
      if (std::fabs(dpn) > 1.0e-30) {
        double den = std::max(dot3(d, d), 1.0e-30);
        double lam = dot3(sub3(m.xf[f], m.cc[Pc]), d) / den;
        lam = std::min(1.0, std::max(0.0, lam));
        double rAUf = (1.0 - lam) * rau[Pc] + lam * rau[N];
        double gx = (1.0 - lam) * g.x[Pc] + lam * g.x[N], gy = (1.0 - lam) * g.y[Pc] + lam * g.y[N],
               gz = (1.0 - lam) * g.z[Pc] + lam * g.z[N];
        double tx = m.Sf[f][0] - (m.Af[f] / dpn) * d[0], ty = m.Sf[f][1] - (m.Af[f] / dpn) * d[1],
               tz = m.Sf[f][2] - (m.Af[f] / dpn) * d[2];
        flux = rAUf * (gx * tx + gy * ty + gz * tz);
        divNO[Pc] += flux;
        divNO[N] += -flux;
      }
    } else {
      int patch = m.bPatch[f] - 1;
      if (patch >= 0 && m.type[3][patch] == 1) {
        int Pc = m.owner[f];
        V3 d = sub3(m.xf[f], m.cc[Pc]);
        double dpn = dot3(m.nf[f], d);
        if (std::fabs(dpn) > 1.0e-30) {
          double tx = m.Sf[f][0] - (m.Af[f] / dpn) * d[0], ty = m.Sf[f][1] - (m.Af[f] / dpn) * d[1],
                 tz = m.Sf[f][2] - (m.Af[f] / dpn) * d[2];
          flux = rau[Pc] * (g.x[Pc] * tx + g.y[Pc] * ty + g.z[Pc] * tz);
          divNO[Pc] += flux;
        }
      }
    }
    phiNO[f] = flux;
  }
}

// kernel_correct_face_fluxes_simple_nonorth, GSV1:1615-1658.
void flux_correct(const orc_mesh& m, const double* rau, const std::vector<double>& phiStar, const double* pc,
                  const std::vector<double>& phiNO, std::vector<double>& phi) {
#pragma omp parallel for schedule(static)
  for (int f = 0; f < m.nFaces; ++f) {
    if (f < m.nInternal) {
      int Pc = m.owner[f], N = m.neigh[f];
      V3 d = sub3(m.cc[N], m.cc[Pc]);
      double dpn = dot3(m.nf[f], d);
      double den = std::max(dot3(d, d), 1.0e-30);
      double lam = dot3(sub3(m.xf[f], m.cc[Pc]), d) / den;
      lam = std::min(1.0, std::max(0.0, lam));
      double rAUf = (1.0 - lam) * rau[Pc] + lam * rau[N];
      double coeff = m.Af[f] * rAUf / dpn;
      phi[f] = phiStar[f] - coeff * (pc[N] - pc[Pc]) - phiNO[f];
    } else {
      int patch = m.bPatch[f] - 1;
      if (patch >= 0 && m.type[3][patch] == 1) {
        int Pc = m.owner[f];
        V3 d = sub3(m.xf[f], m.cc[Pc]);
        double dpn = dot3(m.nf[f], d);
        if (std::fabs(dpn) <= 1.0e-30) {
          phi[f] = phiStar[f];
          continue;
        }
        double coeff = m.Af[f] * rau[Pc] / dpn;
        phi[f] = phiStar[f] - coeff * (m.fval[3][f] - pc[Pc]) - phiNO[f];
      } else {
        phi[f] = phiStar[f];
      }
    }
  }
}

// ---- deterministic FP64 Krylov solvers standing in for HYPRE (GSV1:2553-2676) ----
void spmv(const CSR& A, const std::vector<double>& vals, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int r = 0; r < A.n; ++r) {
    double s = 0.0;
    for (int k = A.rowOff[r]; k < A.rowOff[r + 1]; ++k) s += vals[k] * x[A.cols[k]];
    y[r] = s;
  }
}

// Right-Jacobi-preconditioned BiCGSTAB; stop when ||r||_2 <= max(atol, rtol*||b||).
int bicgstab(const CSR& A, const std::vector<double>& vals, const std::vector<double>& b, std::vector<double>& x,
             double atol, double rtol, int maxit, bool* conv) {
  const int n = A.n;
  std::vector<double> dinv(n), r(n), rh(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
  for (int i = 0; i < n; ++i) {
    double d = vals[A.diagPos[i]];
    dinv[i] = d != 0.0 ? 1.0 / d : 1.0;
  }
  spmv(A, vals, x.data(), r.data());
  for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
  rh = r;
  double bn = std::sqrt(det_sum(n, [&](int i) { return b[i] * b[i]; }));
  double eps = std::max(atol, rtol * bn);
  double rn = std::sqrt(det_sum(n, [&](int i) { return r[i] * r[i]; }));
  *conv = true;
  if (rn <= eps) return 0;
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  int it = 0;
  while (it < maxit) {
    ++it;
    double rhoN = det_sum(n, [&](int i) { return rh[i] * r[i]; });
    double beta = (rhoN / rho) * (alpha / omega);
    rho = rhoN;
    for (int i = 0; i < n; ++i) {
      p[i] = r[i] + beta * (p[i] - omega * v[i]);
      ph[i] = dinv[i] * p[i];
    }
    spmv(A, vals, ph.data(), v.data());
    alpha = rho / det_sum(n, [&](int i) { return rh[i] * v[i]; });
    for (int i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
    double sn = std::sqrt(det_sum(n, [&](int i) { return s[i] * s[i]; }));
    if (sn <= eps) {
      for (int i = 0; i < n; ++i) x[i] += alpha * ph[i];
      return it;
    }
    for (int i = 0; i < n; ++i) sh[i] = dinv[i] * s[i];
    spmv(A, vals, sh.data(), t.data());
    double ts = det_sum(n, [&](int i) { return t[i] * s[i]; });
    double tt = det_sum(n, [&](int i) { return t[i] * t[i]; });
    omega = tt > 0 ? ts / tt : 0.0;
    for (int i = 0; i < n; ++i) {
      x[i] += alpha * ph[i] + omega * sh[i];
      r[i] = s[i] - omega * t[i];
    }
    rn = std::sqrt(det_sum(n, [&](int i) { return r[i] * r[i]; }));
    if (rn <= eps) return it;
    if (omega == 0.0) break;
  }
  *conv = false;
  return it;
}

// ---- aggregation AMG for the CPU pressure solve (stand-in for the reference's BoomerAMG, ----
// GSV1:2242-2260; an implementation of its own, not the B200 library's).  Rebuilt from every outer
// step's pressure matrix, as the reference rebuilds its hierarchy at pAmgRebuildEvery = 1
// (GSV1:3409-3411): greedy aggregation on strong negative couplings (-a_ij >= 0.25 max_k -a_ik; a
// row and its free strong neighbours form an aggregate, leftover rows join their strongest
// neighbour's), piecewise-constant prolongation, Galerkin coarse operators down to <= 200 rows,
// Cholesky there; a symmetric V(1,1) cycle with weighted Jacobi (0.9) and the coarse correction
// scaled by 1.6 (over-correction keeps it SPD).  Used by the timed CPU baseline (p_use_amg).
struct AmgLev {
  int n = 0, nc = 0;
  std::vector<int> off, col;     // CSR, diagonal included
  std::vector<double> val, diag;
  std::vector<int> agg, memOff, mem;
  std::vector<double> b, x, r;
};
struct CpuAmg {
  std::vector<AmgLev> lv;
  std::vector<double> L;  // Cholesky factor of the coarsest level (row-major, lower)
  std::vector<char> skip;
};

void amg_build(const CSR& A, const std::vector<double>& vals, CpuAmg& H) {
  H.lv.clear();
  AmgLev l0;
  l0.n = A.n;
  l0.off = A.rowOff;
  l0.col = A.cols;
  l0.val = vals;
  H.lv.push_back(std::move(l0));
  for (;;) {
    AmgLev& f = H.lv.back();
    const int n = f.n;
    f.diag.assign(n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int k = f.off[i]; k < f.off[i + 1]; ++k)
        if (f.col[k] == i) f.diag[i] = f.val[k];
    f.b.assign(n, 0.0);
    f.x.assign(n, 0.0);
    f.r.assign(n, 0.0);
    if (n <= 200 || H.lv.size() >= 20) break;
    std::vector<double> mx(n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int k = f.off[i]; k < f.off[i + 1]; ++k)
        if (f.col[k] != i) mx[i] = std::max(mx[i], -f.val[k]);
    auto strong = [&](int i, int k) { return f.col[k] != i && -f.val[k] > 0.0 && -f.val[k] >= 0.25 * mx[i]; };
    f.agg.assign(n, -1);
    int nc = 0;
    for (int i = 0; i < n; ++i) {
      if (f.agg[i] >= 0) continue;
      bool free = true;
      for (int k = f.off[i]; k < f.off[i + 1] && free; ++k)
        if (strong(i, k) && f.agg[f.col[k]] >= 0) free = false;
      if (!free) continue;
      f.agg[i] = nc;
      for (int k = f.off[i]; k < f.off[i + 1]; ++k)
        if (strong(i, k)) f.agg[f.col[k]] = nc;
      ++nc;
    }
    std::vector<int> first(f.agg);
    for (int i = 0; i < n; ++i) {
      if (first[i] >= 0) continue;
      int best = -1;
      double bv = 0.0;
      for (int k = f.off[i]; k < f.off[i + 1]; ++k)
        if (strong(i, k) && first[f.col[k]] >= 0 && -f.val[k] > bv) {
          bv = -f.val[k];
          best = first[f.col[k]];
        }
      f.agg[i] = best >= 0 ? best : nc++;
    }
    if (nc > 0.9 * n) break;  // coarsening stalled: this level is the coarsest
    f.nc = nc;
    f.memOff.assign(nc + 1, 0);
    for (int i = 0; i < n; ++i) f.memOff[f.agg[i] + 1]++;
    for (int I = 0; I < nc; ++I) f.memOff[I + 1] += f.memOff[I];
    f.mem.assign(n, 0);
    {
      std::vector<int> fill(f.memOff.begin(), f.memOff.end() - 1);
      for (int i = 0; i < n; ++i) f.mem[fill[f.agg[i]]++] = i;
    }
    AmgLev c;
    c.n = nc;
    c.off.assign(nc + 1, 0);
    std::vector<int> mark(nc, -1), pos(nc, 0);
    for (int I = 0; I < nc; ++I) {
      const size_t start = c.col.size();
      for (int m = f.memOff[I]; m < f.memOff[I + 1]; ++m) {
        const int i = f.mem[m];
        for (int k = f.off[i]; k < f.off[i + 1]; ++k) {
          const int J = f.agg[f.col[k]];
          if (mark[J] != I) {
            mark[J] = I;
            pos[J] = (int)c.col.size();
            c.col.push_back(J);
            c.val.push_back(0.0);
          }
          c.val[pos[J]] += f.val[k];
        }
      }
      c.off[I + 1] = (int)c.col.size();
      (void)start;
    }
    H.lv.push_back(std::move(c));
  }
  // Cholesky of the coarsest level; a pivot below 1e-13 of the largest diagonal (a singular,
  // all-Neumann system) drops its row and column
  const AmgLev& d = H.lv.back();
  const int nd = d.n;
  std::vector<double> M((size_t)nd * nd, 0.0);
  double dm = 0.0;
  for (int i = 0; i < nd; ++i) {
    for (int k = d.off[i]; k < d.off[i + 1]; ++k) M[(size_t)i * nd + d.col[k]] += d.val[k];
    dm = std::max(dm, std::fabs(d.diag[i]));
  }
  H.L.assign((size_t)nd * nd, 0.0);
  H.skip.assign(nd, 0);
  for (int j = 0; j < nd; ++j) {
    double s = M[(size_t)j * nd + j];
    for (int k = 0; k < j; ++k) s -= H.L[(size_t)j * nd + k] * H.L[(size_t)j * nd + k];
    if (s <= 1e-13 * dm) {
      H.skip[j] = 1;
      continue;
    }
    const double ljj = std::sqrt(s);
    H.L[(size_t)j * nd + j] = ljj;
    for (int i = j + 1; i < nd; ++i) {
      double t = M[(size_t)i * nd + j];
      for (int k = 0; k < j; ++k) t -= H.L[(size_t)i * nd + k] * H.L[(size_t)j * nd + k];
      H.L[(size_t)i * nd + j] = t / ljj;
    }
  }
}

void amg_vcycle(CpuAmg& H, size_t l) {
  AmgLev& f = H.lv[l];
  const int n = f.n;
  if (l + 1 == H.lv.size()) {  // coarsest: L L^T x = b
    std::vector<double>& y = f.x;
    for (int i = 0; i < n; ++i) {
      if (H.skip[i]) { y[i] = 0.0; continue; }
      double s = f.b[i];
      for (int k = 0; k < i; ++k) s -= H.L[(size_t)i * n + k] * y[k];
      y[i] = s / H.L[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      if (H.skip[i]) { y[i] = 0.0; continue; }
      double s = y[i];
      for (int k = i + 1; k < n; ++k) s -= H.L[(size_t)k * n + i] * y[k];
      y[i] = s / H.L[(size_t)i * n + i];
    }
    return;
  }
  const double w = 0.9, corr = 1.6;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) f.x[i] = w * f.b[i] / f.diag[i];
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = f.off[i]; k < f.off[i + 1]; ++k) s += f.val[k] * f.x[f.col[k]];
    f.r[i] = f.b[i] - s;
  }
  AmgLev& c = H.lv[l + 1];
#pragma omp parallel for schedule(static)
  for (int I = 0; I < f.nc; ++I) {
    double s = 0.0;
    for (int m = f.memOff[I]; m < f.memOff[I + 1]; ++m) s += f.r[f.mem[m]];
    c.b[I] = s;
  }
  amg_vcycle(H, l + 1);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) f.x[i] += corr * c.x[f.agg[i]];
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = f.off[i]; k < f.off[i + 1]; ++k) s += f.val[k] * f.x[f.col[k]];
    f.r[i] = f.b[i] - s;
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) f.x[i] += w * f.r[i] / f.diag[i];
}

// z = M^-1 r: Jacobi, or one V-cycle of the hierarchy when given
void precondition(CpuAmg* amg, const std::vector<double>& dinv, const std::vector<double>& r, std::vector<double>& z) {
  const int n = (int)r.size();
  if (!amg) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) z[i] = dinv[i] * r[i];
    return;
  }
  AmgLev& f = amg->lv[0];
  std::copy(r.begin(), r.end(), f.b.begin());
  amg_vcycle(*amg, 0);
  std::copy(f.x.begin(), f.x.end(), z.begin());
}

// Preconditioned CG (Jacobi, or the AMG V-cycle above); stop when ||r||_2 <= max(atol, rtol*||b||).
int pcg(const CSR& A, const std::vector<double>& vals, const std::vector<double>& b, std::vector<double>& x,
        double atol, double rtol, int maxit, bool* conv, CpuAmg* amg = nullptr) {
  const int n = A.n;
  std::vector<double> dinv(n), r(n), z(n), p(n), q(n);
  for (int i = 0; i < n; ++i) {
    double d = vals[A.diagPos[i]];
    dinv[i] = d != 0.0 ? 1.0 / d : 1.0;
  }
  spmv(A, vals, x.data(), r.data());
  for (int i = 0; i < n; ++i) r[i] = b[i] - r[i];
  double bn = std::sqrt(det_sum(n, [&](int i) { return b[i] * b[i]; }));
  double eps = std::max(atol, rtol * bn);
  double rr = det_sum(n, [&](int i) { return r[i] * r[i]; });
  *conv = true;
  if (std::sqrt(rr) <= eps) return 0;
  precondition(amg, dinv, r, z);
  for (int i = 0; i < n; ++i) p[i] = z[i];
  double rz = det_sum(n, [&](int i) { return r[i] * z[i]; });
  int it = 0;
  while (it < maxit) {
    ++it;
    spmv(A, vals, p.data(), q.data());
    double alpha = rz / det_sum(n, [&](int i) { return p[i] * q[i]; });
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
    rr = det_sum(n, [&](int i) { return r[i] * r[i]; });
    if (std::sqrt(rr) <= eps) return it;
    precondition(amg, dinv, r, z);
    double rzN = det_sum(n, [&](int i) { return r[i] * z[i]; });
    double beta = rzN / rz;
    rz = rzN;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  *conv = false;
  return it;
}

double relchg(const std::vector<double>& a, const std::vector<double>& b) {
  double num = 0.0, den = 1.0;
  for (size_t i = 0; i < a.size(); ++i) {
    double d = a[i] - b[i];
    num += d * d;
    den += a[i] * a[i];
  }
  return std::sqrt(num / den);
}

}  // namespace

extern "C" {

orc_mesh* orc_mesh_create(int nP, const double* pts, int nF, const int* fo, const int* fp, int nI, const int* own,
                          const int* nei, int nPatch, const int* ps, const int* pn, char* err, int errlen) {
  try {
    orc_mesh* m = new orc_mesh();
    m->P.resize(nP);
    for (int i = 0; i < nP; ++i) m->P[i] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    m->faces.resize(nF);
    for (int f = 0; f < nF; ++f) m->faces[f].assign(fp + fo[f], fp + fo[f + 1]);
    m->owner.assign(own, own + nF);
    m->neigh.assign(nei, nei + nI);
    m->nFaces = nF;
    m->nInternal = nI;
    m->bPatch.assign(nF, 0);
    m->patchStart.assign(ps, ps + nPatch);
    m->patchN.assign(pn, pn + nPatch);
    for (int k = 0; k < nPatch; ++k)
      for (int f = ps[k]; f < ps[k] + pn[k]; ++f) m->bPatch[f] = k + 1;
    build_geometry(*m);
    build_lsq(*m);
    build_pattern(*m);
    for (int q = 0; q < 4; ++q) {
      m->type[q].assign(nPatch, 0);
      m->fval[q].assign(nF, 0.0);
    }
    return m;
  } catch (const std::exception& e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return nullptr;
  }
}

void orc_mesh_free(orc_mesh* m) { delete m; }
int orc_mesh_ncells(const orc_mesh* m) { return m->nCells; }

void orc_mesh_sizes(const orc_mesh* m, int* s) {
  size_t nfp = 0;
  for (const auto& f : m->faces) nfp += f.size();
  s[0] = (int)m->P.size();
  s[1] = m->nFaces;
  s[2] = m->nInternal;
  s[3] = m->nCells;
  s[4] = (int)m->patchStart.size();
  s[5] = (int)nfp;
}

void orc_mesh_patches(const orc_mesh* m, int* ps, int* pn) {
  for (size_t k = 0; k < m->patchStart.size(); ++k) {
    if (ps) ps[k] = m->patchStart[k];
    if (pn) pn[k] = m->patchN[k];
  }
}

void orc_mesh_topology(const orc_mesh* m, double* pts, int* fo, int* fp, int* own, int* nei) {
  if (pts)
    for (size_t i = 0; i < m->P.size(); ++i)
      for (int q = 0; q < 3; ++q) pts[3 * i + q] = m->P[i][q];
  int cur = 0;
  for (int f = 0; f < m->nFaces; ++f) {
    if (fo) fo[f] = cur;
    for (int v : m->faces[f]) {
      if (fp) fp[cur] = v;
      ++cur;
    }
  }
  if (fo) fo[m->nFaces] = cur;
  if (own) std::copy(m->owner.begin(), m->owner.end(), own);
  if (nei) std::copy(m->neigh.begin(), m->neigh.end(), nei);
}

void orc_mesh_geometry(const orc_mesh* m, double* cc, double* vol, double* xf, double* nf, double* sf, double* af,
                       double* mx) {
  for (int c = 0; c < m->nCells; ++c) {
    if (cc) for (int k = 0; k < 3; ++k) cc[3 * c + k] = m->cc[c][k];
    if (vol) vol[c] = m->vol[c];
  }
  for (int f = 0; f < m->nFaces; ++f) {
    for (int k = 0; k < 3; ++k) {
      if (xf) xf[3 * f + k] = m->xf[f][k];
      if (nf) nf[3 * f + k] = m->nf[f][k];
      if (sf) sf[3 * f + k] = m->Sf[f][k];
    }
    if (af) af[f] = m->Af[f];
  }
  if (mx) *mx = m->maxNonOrthDeg;
}

void orc_set_bc(orc_mesh* m, const int* tu, const int* tv, const int* tw, const int* tp, const double* uf,
                const double* vf, const double* wf, const double* pf) {
  const int* T[4] = {tu, tv, tw, tp};
  const double* Fv[4] = {uf, vf, wf, pf};
  for (int q = 0; q < 4; ++q) {
    m->type[q].assign(T[q], T[q] + m->patchStart.size());
    m->fval[q].assign(Fv[q], Fv[q] + m->nFaces);
  }
}

void orc_lsq_gradient(const orc_mesh* m, int field, const double* phi, double* gx, double* gy, double* gz) {
  lsq_grad(*m, field, phi, gx, gy, gz);
}

void orc_momentum(const orc_mesh* mc, double rho, double mu, double uRelax, const double* u, const double* v,
                  const double* w, const double* p, double* diag, double* a_pn, double* a_np, double* rhs3,
                  double* rau) {
  orc_mesh& m = const_cast<orc_mesh&>(*mc);
  const int n = m.nCells;
  G3 gp(n);
  lsq_grad(m, 3, p, gp.x.data(), gp.y.data(), gp.z.data());
  const double* q[3] = {u, v, w};
  const double* gpc[3] = {gp.x.data(), gp.y.data(), gp.z.data()};
  std::vector<double> rhs(n), rAU(n);
  for (int comp = 0; comp < 3; ++comp) {
    G3 gq(n);
    lsq_grad(m, comp, q[comp], gq.x.data(), gq.y.data(), gq.z.data());
    if (comp == 0) {
      mom_full(m, rho, mu, q[0], 0, gq, gpc[0], u, v, w, rhs);
      mom_relax(m, uRelax, q[0], rhs);
      extract_rau(m, rAU);
    } else {
      mom_rhs_only(m, rho, mu, uRelax, q[comp], comp, gq, gpc[comp], u, v, w, rhs);
    }
    if (rhs3) std::memcpy(rhs3 + (size_t)comp * n, rhs.data(), sizeof(double) * n);
  }
  for (int c = 0; c < n; ++c) {
    if (diag) diag[c] = m.pat.vals[m.pat.diagPos[c]];
    if (rau) rau[c] = rAU[c];
  }
  for (int f = 0; f < m.nInternal; ++f) {
    if (a_pn) a_pn[f] = m.pat.vals[m.pat.fPN[f]];
    if (a_np) a_np[f] = m.pat.vals[m.pat.fNP[f]];
  }
}

void orc_pressure(const orc_mesh* mc, double rho, const double* u, const double* v, const double* w, const double* p,
                  const double* rau, double* diag, double* a_pn, double* phi_star, double* div_star) {
  const orc_mesh& m = *mc;
  std::vector<double> vals(m.pat.vals.size());
  pressure_matrix(m, rau, vals);
  for (int c = 0; c < m.nCells; ++c)
    if (diag) diag[c] = vals[m.pat.diagPos[c]];
  for (int f = 0; f < m.nInternal; ++f)
    if (a_pn) a_pn[f] = vals[m.pat.fPN[f]];
  G3 gp(m.nCells);
  lsq_grad(m, 3, p, gp.x.data(), gp.y.data(), gp.z.data());
  std::vector<double> ps(m.nFaces), dv(m.nCells);
  rhie_chow(m, rho, u, v, w, p, gp, rau, ps);
  continuity(m, ps, dv);
  if (phi_star) std::memcpy(phi_star, ps.data(), sizeof(double) * m.nFaces);
  if (div_star) std::memcpy(div_star, dv.data(), sizeof(double) * m.nCells);
}

void orc_nonorth(const orc_mesh* m, const double* rau, const double* g, double* phi_no, double* div_no) {
  const int n = m->nCells;
  G3 gg(n);
  for (int c = 0; c < n; ++c) {
    gg.x[c] = g[c];
    gg.y[c] = g[n + c];
    gg.z[c] = g[2 * n + c];
  }
  std::vector<double> a(m->nFaces), b(n);
  nonorth(*m, rau, gg, a, b);
  std::memcpy(phi_no, a.data(), sizeof(double) * m->nFaces);
  std::memcpy(div_no, b.data(), sizeof(double) * n);
}

void orc_flux_correct(const orc_mesh* m, const double* rau, const double* phi_star, const double* pcorr,
                      const double* g, double* phi) {
  const int n = m->nCells;
  G3 gg(n);
  for (int c = 0; c < n; ++c) {
    gg.x[c] = g[c];
    gg.y[c] = g[n + c];
    gg.z[c] = g[2 * n + c];
  }
  std::vector<double> no(m->nFaces), dno(n), ps(phi_star, phi_star + m->nFaces), out(m->nFaces);
  nonorth(*m, rau, gg, no, dno);
  flux_correct(*m, rau, ps, pcorr, no, out);
  std::memcpy(phi, out.data(), sizeof(double) * m->nFaces);
}

// SIMPLE loop, GSV1:3350-3634.
int orc_simple_run(orc_mesh* mp, const orc_params* prm, int nsteps, double* uIO, double* vIO, double* wIO,
                   double* pIO, double* phiOut, orc_stats* stats) {
#ifdef _OPENMP
  if (prm->n_threads > 0) omp_set_num_threads(prm->n_threads);
#endif
  orc_mesh& m = *mp;
  const int n = m.nCells;
  std::vector<double> u(uIO, uIO + n), v(vIO, vIO + n), w(wIO, wIO + n), p(pIO, pIO + n);
  std::vector<double> uOld(n), vOld(n), wOld(n), pOld(n), uS(n), vS(n), wS(n), pCorr(n), rAU(n), rhs(n);
  std::vector<double> phiStar(m.nFaces), phi(m.nFaces), phiNO(m.nFaces), divStar(n), divCorr(n), divNO(n);
  std::vector<double> pvals(m.pat.vals.size());
  CpuAmg amg;  // pressure preconditioner with p_use_amg, rebuilt every outer step
  int done = 0;
  for (int step = 1; step <= nsteps; ++step) {
    uOld = u; vOld = v; wOld = w; pOld = p;
    G3 gp(n);
    lsq_grad(m, 3, pOld.data(), gp.x.data(), gp.y.data(), gp.z.data());
    const std::vector<double>* gpc[3] = {&gp.x, &gp.y, &gp.z};
    std::vector<double>* qs[3] = {&uS, &vS, &wS};
    const std::vector<double>* qo[3] = {&uOld, &vOld, &wOld};
    int its[3] = {0, 0, 0};
    bool anyNC = false;
    for (int comp = 0; comp < 3; ++comp) {  // solve_scalar_component_with_nonorth, GSV1:3350-3384
      std::vector<double> qIter = *qo[comp], qNew = qIter;
      const int nVel = std::max(prm->n_vel_nonorth_corr, 0) + 1;
      for (int it = 1; it <= nVel; ++it) {
        G3 gq(n);
        lsq_grad(m, comp, qIter.data(), gq.x.data(), gq.y.data(), gq.z.data());
        if (comp == 0 && it == 1) {
          mom_full(m, prm->rho, prm->mu, qIter.data(), 0, gq, gpc[0]->data(), uOld.data(), vOld.data(), wOld.data(), rhs);
          mom_relax(m, prm->u_relax, qIter.data(), rhs);
          extract_rau(m, rAU);
        } else {
          mom_rhs_only(m, prm->rho, prm->mu, prm->u_relax, qIter.data(), comp, gq, gpc[comp]->data(), uOld.data(),
                       vOld.data(), wOld.data(), rhs);
        }
        qNew = qIter;
        bool conv = true;
        its[comp] = bicgstab(m.pat, m.pat.vals, rhs, qNew, prm->vel_tol, prm->vel_rel_tol, prm->vel_maxit, &conv);
        anyNC = anyNC || !conv;
        double rc = relchg(qNew, qIter);
        qIter.swap(qNew);
        if (rc < prm->corr_tol) break;
      }
      *qs[comp] = qIter;
    }
    pressure_matrix(m, rAU.data(), pvals);  // GSV1:3407-3411
    if (prm->p_use_amg) amg_build(m.pat, pvals, amg);
    u = uS; v = vS; w = wS; p = pOld;
    lsq_grad(m, 3, p.data(), gp.x.data(), gp.y.data(), gp.z.data());
    rhie_chow(m, prm->rho, u.data(), v.data(), w.data(), p.data(), gp, rAU.data(), phiStar);
    phi = phiStar;
    continuity(m, phi, divCorr);
    divStar = divCorr;
    std::fill(pCorr.begin(), pCorr.end(), 0.0);
    const int nPS = std::max(prm->n_nonorth_corr, 0) + 1, nExtra = std::max(prm->n_pressure_corr, 0);
    const int total = nPS + nExtra;
    int counter = 0, pTot = 0, pLast = 0;
    G3 gc(n);
    std::vector<double> b(n);
    for (int pc = 1; pc <= nPS; ++pc) {
      lsq_grad(m, 3, pCorr.data(), gc.x.data(), gc.y.data(), gc.z.data());
      nonorth(m, rAU.data(), gc, phiNO, divNO);
      for (int c = 0; c < n; ++c) b[c] = -divStar[c] + divNO[c];
      ++counter;
      double rtol = (counter == total) ? 0.0 : prm->p_rel_tol;
      bool conv = true;
      pLast = pcg(m.pat, pvals, b, pCorr, prm->p_tol, rtol, prm->p_maxit, &conv, prm->p_use_amg ? &amg : nullptr);
      anyNC = anyNC || !conv;
      pTot += pLast;
      if (pc == nPS) {
        lsq_grad(m, 3, pCorr.data(), gc.x.data(), gc.y.data(), gc.z.data());
        nonorth(m, rAU.data(), gc, phiNO, divNO);
        flux_correct(m, rAU.data(), phiStar, pCorr.data(), phiNO, phi);
        continuity(m, phi, divCorr);
      }
    }
    for (int pc = 1; pc <= nExtra; ++pc) {  // GSV1:3521-3567
      for (int c = 0; c < n; ++c) b[c] = -divCorr[c];
      std::vector<double> dpc(n, 0.0);
      ++counter;
      double rtol = (counter == total) ? 0.0 : prm->p_rel_tol;
      bool conv = true;
      pLast = pcg(m.pat, pvals, b, dpc, prm->p_tol, rtol, prm->p_maxit, &conv, prm->p_use_amg ? &amg : nullptr);
      anyNC = anyNC || !conv;
      pTot += pLast;
      for (int c = 0; c < n; ++c) pCorr[c] += 1.0 * dpc[c];
      lsq_grad(m, 3, pCorr.data(), gc.x.data(), gc.y.data(), gc.z.data());
      nonorth(m, rAU.data(), gc, phiNO, divNO);
      flux_correct(m, rAU.data(), phiStar, pCorr.data(), phiNO, phi);
      continuity(m, phi, divCorr);
    }
    double massRes = 0.0;
    for (int c = 0; c < n; ++c) massRes = std::max(massRes, std::fabs(divCorr[c]));
    for (int c = 0; c < n; ++c) p[c] += prm->p_relax * pCorr[c];
    lsq_grad(m, 3, pCorr.data(), gc.x.data(), gc.y.data(), gc.z.data());
    for (int c = 0; c < n; ++c) {
      u[c] = uS[c] - rAU[c] * gc.x[c];
      v[c] = vS[c] - rAU[c] * gc.y[c];
      w[c] = wS[c] - rAU[c] * gc.z[c];
    }
    double du = relchg(u, uOld), dv = relchg(v, vOld), dw = relchg(w, wOld), dp = relchg(p, pOld);
    (void)anyNC;
    if (stats) stats[step - 1] = {massRes, du, dv, dw, dp, its[0], its[1], its[2], pLast, pTot};
    done = step;
    if (!std::isfinite(massRes) || massRes > 1e50) break;
    if (massRes < prm->tol_mass && std::max({du, dv, dw}) < prm->tol_vel) break;
  }
  std::memcpy(uIO, u.data(), sizeof(double) * n);
  std::memcpy(vIO, v.data(), sizeof(double) * n);
  std::memcpy(wIO, w.data(), sizeof(double) * n);
  std::memcpy(pIO, p.data(), sizeof(double) * n);
  if (phiOut) std::memcpy(phiOut, phi.data(), sizeof(double) * m.nFaces);
  return done;
}

// compute_patch_forces_wall_shear, GSV1:2828-2933.
void orc_patch_force(const orc_mesh* m, int patch, int sign, double mu, const double* u, const double* v,
                     const double* w, const double* p, double* o) {
  for (int k = 0; k < 11; ++k) o[k] = 0.0;
  double minD = 1.0e300, maxD = 0.0, maxUt = 0.0, maxSh = 0.0;
  int nF = 0;
  const int f0 = m->patchStart[patch], f1 = f0 + m->patchN[patch];
  for (int f = f0; f < f1; ++f) {
    int Pc = m->owner[f];
    double A = m->Af[f];
    if (A <= 1.0e-300) continue;
    V3 nv{(double)sign * m->nf[f][0], (double)sign * m->nf[f][1], (double)sign * m->nf[f][2]};
    double nm = norm3(nv);
    if (nm <= 1.0e-300) continue;
    nv = mul3(1.0 / nm, nv);
    V3 dx = sub3(m->cc[Pc], m->xf[f]);
    double dn = dot3(dx, nv);
    if (dn <= 1.0e-14) dn = std::fabs(dn);
    if (dn <= 1.0e-14) dn = norm3(dx);
    if (dn <= 1.0e-14) continue;
    V3 U{u[Pc], v[Pc], w[Pc]};
    double Un = dot3(U, nv);
    V3 Ut = sub3(U, mul3(Un, nv));
    double Utm = norm3(Ut), sh = mu * Utm / dn;
    for (int d = 0; d < 3; ++d) {
      double fp = -p[Pc] * nv[d] * A, fv = mu * Ut[d] / dn * A;
      o[d] += fp;
      o[3 + d] += fv;
      o[6 + d] += fp + fv;
    }
    o[9] += A;
    ++nF;
    minD = std::min(minD, dn);
    maxD = std::max(maxD, dn);
    maxUt = std::max(maxUt, Utm);
    maxSh = std::max(maxSh, sh);
  }
  o[10] = nF;
  (void)minD; (void)maxD; (void)maxUt; (void)maxSh;
}

/* ---- scalar libraries (libpoisson, libscalar) ------------------------------------------------
 * bc_type per face (boundary entries read): 0 Dirichlet, 1 prescribed normal gradient, 2 zero
 * gradient (libscalar). */

/* compute_lsq_gradient of libpoisson/src/gradient.cu:21-83 (libscalar's copy at
 * scalar_transport_library.cu:185-246 is the same): neighbours as usual, Dirichlet faces at the
 * face centre, other boundary faces as the pure-normal constraint r = dn n, dphi = g dn. */
void orc_scalar_gradient(const orc_mesh* m, const int* bt, const double* bv, const double* phi, double* gx,
                         double* gy, double* gz) {
#pragma omp parallel for schedule(static)
  for (int P = 0; P < m->nCells; ++P) {
    const V3 xP = m->cc[P];
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, b[3] = {0, 0, 0};
    auto acc = [&](const V3& r, double dphi) {
      const double w = 1.0 / std::max(dot3(r, r), 1e-30);
      for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) M[i][j] += w * r[i] * r[j];
        b[i] += w * r[i] * dphi;
      }
    };
    for (int N : m->cellNbrs[P]) acc(sub3(m->cc[N], xP), phi[N] - phi[P]);
    for (int f : m->cellBFace[P]) {
      const V3 rcf = sub3(m->xf[f], xP);
      if (bt[f] == 0) {
        acc(rcf, bv[f] - phi[P]);
      } else {
        const double dn = std::max(dot3(rcf, m->nf[f]), 1e-30);
        acc(mul3(dn, m->nf[f]), bv[f] * dn);
      }
    }
    const double a = M[0][0], bb = M[0][1], c = M[0][2], d = M[1][0], e = M[1][1], f2 = M[1][2], g = M[2][0],
                 h = M[2][1], k = M[2][2];
    const double det = a * (e * k - f2 * h) - bb * (d * k - f2 * g) + c * (d * h - e * g);
    double o[3] = {0, 0, 0};
    if (std::fabs(det) > 1e-20) {
      const double inv[3][3] = {{(e * k - f2 * h) / det, (c * h - bb * k) / det, (bb * f2 - c * e) / det},
                                {(f2 * g - d * k) / det, (a * k - c * g) / det, (c * d - a * f2) / det},
                                {(d * h - e * g) / det, (bb * g - a * h) / det, (a * e - bb * d) / det}};
      for (int i = 0; i < 3; ++i) o[i] = inv[i][0] * b[0] + inv[i][1] * b[1] + inv[i][2] * b[2];
    }
    gx[P] = o[0];
    gy[P] = o[1];
    gz[P] = o[2];
  }
}

/* Assembly in face-coefficient form: diag[C], a_pn[Fi] (row owner, column neighbour),
 * a_np[Fi] (row neighbour, column owner), rhs[C].  transport == 0: libpoisson
 * assemble_scalar_elliptic_system (scalar_elliptic.cu:60-136, reference cell row replaced by the
 * identity as at 126-135); transport == 1: libscalar assemble_scalar_transport_system
 * (scalar_transport_library.cu:250-357).  grad is 3 x nCells SoA; flux/sp may be NULL. */
void orc_scalar_assemble(const orc_mesh* m, int transport, int upwind, int nonorth, const double* gamma,
                         const double* flux, const double* src, const double* sp, const int* bt, const double* bv,
                         const double* grad, int ref_cell, double ref_value, double* diag, double* a_pn,
                         double* a_np, double* rhs) {
  const int C = m->nCells, nI = m->nInternal;
  const double *gx = grad, *gy = grad + C, *gz = grad + 2 * C;
  for (int c = 0; c < C; ++c) {
    rhs[c] = src[c] * m->vol[c];
    diag[c] = (transport && sp) ? -sp[c] * m->vol[c] : 0.0;
  }
  for (int f = 0; f < nI; ++f) {
    const int P = m->owner[f], N = m->neigh[f];
    const V3 d = sub3(m->cc[N], m->cc[P]);
    const double D = gamma[f] * dot3(m->Sf[f], m->Sf[f]) / std::max(dot3(d, m->Sf[f]), 1e-30);
    diag[P] += D;
    diag[N] += D;
    a_pn[f] = -D;
    a_np[f] = -D;
    const V3 dx = sub3(m->xf[f], m->cc[P]);
    const double lam = std::min(1.0, std::max(0.0, dot3(dx, d) / std::max(dot3(d, d), 1e-30)));
    if (nonorth) {
      const V3 T = sub3(m->Sf[f], mul3(D / std::max(gamma[f], 1e-30), d));
      const V3 gf{(1.0 - lam) * gx[P] + lam * gx[N], (1.0 - lam) * gy[P] + lam * gy[N],
                  (1.0 - lam) * gz[P] + lam * gz[N]};
      const double corr = gamma[f] * dot3(T, gf);
      rhs[P] += corr;
      rhs[N] -= corr;
    }
    if (transport && flux) {
      const double F = flux[f];
      if (!upwind) {
        diag[P] += F * (1.0 - lam);
        a_pn[f] += F * lam;
        a_np[f] -= F * (1.0 - lam);
        diag[N] -= F * lam;
      } else if (F >= 0.0) {
        diag[P] += F;
        a_np[f] -= F;
      } else {
        a_pn[f] += F;
        diag[N] -= F;
      }
    }
  }
  for (int f = nI; f < m->nFaces; ++f) {
    const int P = m->owner[f];
    const V3 d = sub3(m->xf[f], m->cc[P]);
    const double D = gamma[f] * dot3(m->Sf[f], m->Sf[f]) / std::max(dot3(d, m->Sf[f]), 1e-30);
    const double F = (transport && flux) ? flux[f] : 0.0;
    if (bt[f] == 0) {
      diag[P] += D;
      rhs[P] += D * bv[f];
      if (nonorth) {
        const V3 T = sub3(m->Sf[f], mul3(D / std::max(gamma[f], 1e-30), d));
        rhs[P] += gamma[f] * (T[0] * gx[P] + T[1] * gy[P] + T[2] * gz[P]);
      }
      if (transport) rhs[P] += -F * bv[f];
    } else if (transport) {
      rhs[P] += gamma[f] * (bt[f] == 2 ? 0.0 : bv[f]) * m->Af[f];
      diag[P] += F;
    } else {
      rhs[P] += -gamma[f] * bv[f] * m->Af[f];
    }
  }
  if (ref_cell >= 0 && ref_cell < C) {
    for (int f = 0; f < nI; ++f) {
      if (m->owner[f] == ref_cell) a_pn[f] = 0.0;
      if (m->neigh[f] == ref_cell) a_np[f] = 0.0;
    }
    diag[ref_cell] = 1.0;
    rhs[ref_cell] = ref_value;
  }
}

}  // extern "C"
