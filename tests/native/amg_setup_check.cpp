// CPU check of the AMG hierarchy set-up (anabasis_b200/csrc/amg_setup.cpp), no GPU needed.
//
// Builds the hierarchy of a random symmetric M-matrix on an NX x NY x NZ 7-point grid twice: with
// the coarse levels above `sellMinRows` rows stored SELL-32 and with every coarse level CSR.  For
// each level it recomputes the coarse values through the Galerkin gather lists (what
// k_amg_galerkin does on the device), checks every index against its array, checks that each row
// belongs to exactly one aggregate, and compares y = A x of both storage forms on a random x.
// Prints one line per level and "OK" at the end; exits non-zero on the first failure.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "amg_setup.hpp"

using namespace anb;

namespace {

int fail(const char* what, size_t level) {
  std::printf("FAIL level %zu: %s\n", level, what);
  return 1;
}

bool gather(const AmgLevelHost& f, const AmgLevelHost& c, const std::vector<double>& val, const std::vector<double>& diag,
            std::vector<double>& valNext, std::vector<double>& diagNext) {
  const int nT = c.nStore + c.n;
  if ((int)f.gOff.size() != nT + 1) return false;
  valNext.assign(c.nStore, 0.0);
  diagNext.assign(c.n, 0.0);
  for (int t = 0; t < nT; ++t) {
    double s = 0.0;
    for (int k = f.gOff[t]; k < f.gOff[t + 1]; ++k) {
      const int idx = f.gIdx[k];
      if (idx >= 0) {
        if (idx >= (int)val.size()) return false;
        s += val[idx];
      } else {
        if (-1 - idx >= (int)diag.size()) return false;
        s += diag[-1 - idx];
      }
    }
    (t < c.nStore ? valNext[t] : diagNext[t - c.nStore]) = s;
  }
  return true;
}

bool spmv(const AmgLevelHost& h, const std::vector<double>& val, const std::vector<double>& diag,
          const std::vector<double>& x, std::vector<double>& y) {
  y.assign(h.n, 0.0);
  for (int i = 0; i < h.n; ++i) {
    double acc = diag[i] * x[i];
    if (!h.sliceOff.empty()) {
      const int s = i / kSlice, w = (h.sliceOff[s + 1] - h.sliceOff[s]) / kSlice;
      if (w > h.maxW) return false;
      for (int k = 0; k < w; ++k) {
        const int e = h.sliceOff[s] + kSlice * k + i % kSlice;
        if (e >= h.nStore || h.col[e] < 0 || h.col[e] >= h.n) return false;
        acc += val[e] * x[h.col[e]];
      }
    } else {
      if ((int)h.rowOff.size() != h.n + 1 || h.rowOff[h.n] != h.nStore) return false;
      for (int k = h.rowOff[i]; k < h.rowOff[i + 1]; ++k) {
        if (h.col[k] < 0 || h.col[k] >= h.n || h.col[k] == i) return false;
        acc += val[k] * x[h.col[k]];
      }
    }
    y[i] = acc;
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  const int NX = argc > 1 ? std::atoi(argv[1]) : 40, NY = argc > 2 ? std::atoi(argv[2]) : 40,
            NZ = argc > 3 ? std::atoi(argv[3]) : 20, sellMin = argc > 4 ? std::atoi(argv[4]) : 1000;
  const int C = NX * NY * NZ;
  auto id = [&](int i, int j, int k) { return (k * NY + j) * NX + i; };
  std::vector<std::vector<int>> nb(C);
  for (int k = 0; k < NZ; ++k)
    for (int j = 0; j < NY; ++j)
      for (int i = 0; i < NX; ++i) {
        auto& v = nb[id(i, j, k)];
        if (k > 0) v.push_back(id(i, j, k - 1));
        if (j > 0) v.push_back(id(i, j - 1, k));
        if (i > 0) v.push_back(id(i - 1, j, k));
        if (i + 1 < NX) v.push_back(id(i + 1, j, k));
        if (j + 1 < NY) v.push_back(id(i, j + 1, k));
        if (k + 1 < NZ) v.push_back(id(i, j, k + 1));
      }
  Layout L;
  L.nCells = C;
  L.nSlices = (C + kSlice - 1) / kSlice;
  L.rowLen.resize(C);
  L.sliceOff.assign(L.nSlices + 1, 0);
  for (int r = 0; r < C; ++r) L.rowLen[r] = (int)nb[r].size();
  for (int s = 0; s < L.nSlices; ++s) {
    int w = 0;
    for (int r = s * kSlice; r < std::min(C, (s + 1) * kSlice); ++r) w = std::max(w, L.rowLen[r]);
    L.maxRowLen = std::max(L.maxRowLen, w);
    L.sliceOff[s + 1] = L.sliceOff[s] + w * kSlice;
  }
  auto slot = [&](int r, int k) { return L.sliceOff[r / kSlice] + kSlice * k + r % kSlice; };
  L.col.assign(L.sliceOff.back(), 0);
  std::vector<double> val(L.sliceOff.back(), 0.0), diag(C, 0.1);
  for (int r = 0; r < C; ++r)
    for (int k = 0; k < (L.sliceOff[r / kSlice + 1] - L.sliceOff[r / kSlice]) / kSlice; ++k)
      L.col[slot(r, k)] = k < L.rowLen[r] ? nb[r][k] : r;
  std::mt19937 g(7);
  std::uniform_real_distribution<double> U(0.5, 1.5);
  for (int r = 0; r < C; ++r)
    for (int k = 0; k < L.rowLen[r]; ++k) {
      const int c = nb[r][k];
      if (c < r) continue;
      const double a = -U(g);
      val[slot(r, k)] = a;
      for (int k2 = 0; k2 < L.rowLen[c]; ++k2)
        if (nb[c][k2] == r) val[slot(c, k2)] = a;
      diag[r] -= a;
      diag[c] -= a;
    }

  AmgSetupOptions sell, csr;
  sell.sellMinRows = sellMin;
  csr.sellMinRows = 1 << 30;
  const auto HS = build_amg_hierarchy(L, val, diag, sell);
  const auto HC = build_amg_hierarchy(L, val, diag, csr);
  if (HS.size() != HC.size() || HS.size() < 3) return fail("level count", 0);
  int nSell = 0;
  std::vector<double> vs = val, vc = val, ds = diag, dc = diag;
  for (size_t l = 0; l + 1 < HS.size(); ++l) {
    const AmgLevelHost& f = HS[l];
    if (f.agg != HC[l].agg) return fail("aggregates differ between storage forms", l);
    if ((int)f.agg.size() != f.n || (int)f.memOff.size() != f.nc + 1 || (int)f.mem.size() != f.n)
      return fail("aggregate array sizes", l);
    std::vector<int> seen(f.n, 0);
    for (int I = 0; I < f.nc; ++I)
      for (int mm = f.memOff[I]; mm < f.memOff[I + 1]; ++mm) {
        const int i = f.mem[mm];
        if (i < 0 || i >= f.n || f.agg[i] != I || seen[i]++) return fail("member lists", l);
      }
    std::vector<double> vs2, ds2, vc2, dc2;
    if (!gather(f, HS[l + 1], vs, ds, vs2, ds2) || !gather(HC[l], HC[l + 1], vc, dc, vc2, dc2))
      return fail("gather list index out of range", l);
    vs = vs2, ds = ds2, vc = vc2, dc = dc2;
    const AmgLevelHost& c = HS[l + 1];
    nSell += !c.sliceOff.empty();
    std::vector<double> x(c.n), ys, yc;
    for (double& v : x) v = U(g);
    if (!spmv(c, vs, ds, x, ys) || !spmv(HC[l + 1], vc, dc, x, yc)) return fail("coarse pattern index out of range", l + 1);
    double md = 0.0, my = 0.0;
    for (int i = 0; i < c.n; ++i) {
      md = std::max(md, std::fabs(ys[i] - yc[i]));
      my = std::max(my, std::fabs(yc[i]));
    }
    std::printf("level %zu rows %d %s slots %d max|dy| %.3e\n", l + 1, c.n, c.sliceOff.empty() ? "CSR " : "SELL",
                c.nStore, md);
    if (md > 1e-12 * my) return fail("SELL and CSR operators differ", l + 1);
  }
  if (nSell == 0) return fail("no SELL level exercised", 0);
  std::printf("OK\n");
  return 0;
}
