// Aggregation AMG structure set-up (host).
#include "amg_setup.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace anb {
namespace {

// Plain CSR with diagonal separate; entry ids refer back to the fine storage for gathers.
struct HCsr {
  int n = 0;
  std::vector<int> off, col;
  std::vector<double> val, diag;
};

// One pass of pairwise aggregation by heavy-edge matching: edges (i, j) with negative coupling,
// strength -a_ij / sqrt(a_ii a_jj), are visited strongest first and matched when both ends are
// free and the edge is strong for either end (>= beta of that row's strongest coupling).  Rows
// left unmatched join the aggregate of their strongest neighbour (aggregates of 2-3 rows), or
// stay single when they have no negative coupling.  Ties break on row index, so the result is
// deterministic.  Returns the aggregate of every row; nc receives the aggregate count, numbered
// in order of each aggregate's first row.
std::vector<int> pairwise(const HCsr& A, double beta, int& nc) {
  const int n = A.n;
  std::vector<double> rowMax(n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = A.off[i]; k < A.off[i + 1]; ++k) rowMax[i] = std::max(rowMax[i], -A.val[k]);
  struct Edge {
    double s;
    int i, j;
  };
  std::vector<Edge> edges;
  edges.reserve(A.off[n] / 2 + 1);
  for (int i = 0; i < n; ++i)
    for (int k = A.off[i]; k < A.off[i + 1]; ++k) {
      const int j = A.col[k];
      const double a = -A.val[k];
      if (j <= i || a <= 0.0) continue;
      if (a < beta * rowMax[i] && a < beta * rowMax[j]) continue;
      const double dd = std::sqrt(std::max(A.diag[i], 1e-300) * std::max(A.diag[j], 1e-300));
      edges.push_back({a / dd, i, j});
    }
  std::sort(edges.begin(), edges.end(), [](const Edge& x, const Edge& y) {
    if (x.s != y.s) return x.s > y.s;
    if (x.i != y.i) return x.i < y.i;
    return x.j < y.j;
  });
  std::vector<int> mate(n, -1);
  for (const Edge& e : edges)
    if (mate[e.i] < 0 && mate[e.j] < 0) {
      mate[e.i] = e.j;
      mate[e.j] = e.i;
    }
  std::vector<int> agg(n, -1);
  nc = 0;
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0 || mate[i] < 0) continue;
    agg[i] = agg[mate[i]] = nc++;
  }
  for (int i = 0; i < n; ++i) {
    if (mate[i] >= 0) continue;
    int best = -1;
    double bestV = 0.0;
    for (int k = A.off[i]; k < A.off[i + 1]; ++k) {
      const int j = A.col[k];
      const double a = -A.val[k];
      if (j == i || a <= 0.0 || mate[j] < 0) continue;
      if (best < 0 || a > bestV) {
        best = j;
        bestV = a;
      }
    }
    agg[i] = best >= 0 ? agg[best] : -2;
  }
  for (int i = 0; i < n; ++i)
    if (agg[i] == -2) agg[i] = nc++;
  // renumber aggregates in order of their first row (keeps the coarse ordering banded)
  std::vector<int> ren(nc, -1);
  int next = 0;
  for (int i = 0; i < n; ++i) {
    if (ren[agg[i]] < 0) ren[agg[i]] = next++;
    agg[i] = ren[agg[i]];
  }
  return agg;
}

// Galerkin product with piecewise-constant prolongation.
HCsr galerkin(const HCsr& A, const std::vector<int>& agg, int nc) {
  HCsr C;
  C.n = nc;
  C.diag.assign(nc, 0.0);
  std::vector<std::vector<std::pair<int, double>>> rows(nc);
  for (int i = 0; i < A.n; ++i) {
    const int I = agg[i];
    C.diag[I] += A.diag[i];
    for (int k = A.off[i]; k < A.off[i + 1]; ++k) {
      const int J = agg[A.col[k]];
      if (J == I) {
        C.diag[I] += A.val[k];
        continue;
      }
      auto& r = rows[I];
      auto it = std::find_if(r.begin(), r.end(), [J](const std::pair<int, double>& p) { return p.first == J; });
      if (it == r.end()) r.push_back({J, A.val[k]});
      else it->second += A.val[k];
    }
  }
  C.off.assign(nc + 1, 0);
  for (int I = 0; I < nc; ++I) {
    std::sort(rows[I].begin(), rows[I].end());
    C.off[I + 1] = C.off[I] + (int)rows[I].size();
  }
  C.col.resize(C.off[nc]);
  C.val.resize(C.off[nc]);
  for (int I = 0; I < nc; ++I)
    for (size_t k = 0; k < rows[I].size(); ++k) {
      C.col[C.off[I] + k] = rows[I][k].first;
      C.val[C.off[I] + k] = rows[I][k].second;
    }
  return C;
}

}  // namespace

std::vector<AmgLevelHost> build_amg_hierarchy(const Layout& L, const std::vector<double>& vals,
                                              const std::vector<double>& diag, const AmgSetupOptions& opt) {
  std::vector<AmgLevelHost> levels;
  // level 0 as CSR, remembering each CSR entry's SELL storage index
  HCsr A;
  A.n = L.nCells;
  A.off.assign(A.n + 1, 0);
  for (int r = 0; r < A.n; ++r) A.off[r + 1] = A.off[r] + L.rowLen[r];
  A.col.resize(A.off[A.n]);
  A.val.resize(A.off[A.n]);
  A.diag = diag;
  std::vector<int> storage(A.off[A.n]);
  for (int r = 0; r < A.n; ++r) {
    const int s = r / kSlice, lane = r % kSlice;
    for (int k = 0; k < L.rowLen[r]; ++k) {
      const int e = L.sliceOff[s] + k * kSlice + lane;
      A.col[A.off[r] + k] = L.col[e];
      A.val[A.off[r] + k] = vals[e];
      storage[A.off[r] + k] = e;
    }
  }
  {
    AmgLevelHost lv0;
    lv0.n = A.n;
    lv0.nStore = L.sliceOff.back();
    lv0.maxW = L.maxRowLen;
    levels.push_back(std::move(lv0));  // pattern comes from the mesh layout
  }
  while ((int)levels.size() < opt.maxLevels && A.n > opt.coarseMax) {
    // aggregates = composition of pairwise passes
    std::vector<int> agg(A.n);
    for (int i = 0; i < A.n; ++i) agg[i] = i;
    int nc = A.n;
    HCsr B = A;
    const size_t lev = levels.size() - 1;
    const int nPass = opt.passes.empty() ? opt.passesPerLevel
                                         : opt.passes[std::min(lev, opt.passes.size() - 1)];
    for (int pass = 0; pass < nPass; ++pass) {
      int ncp = 0;
      std::vector<int> a = pairwise(B, opt.strength, ncp);
      for (int i = 0; i < A.n; ++i) agg[i] = a[agg[i]];
      nc = ncp;
      if (pass + 1 < nPass) B = galerkin(B, a, ncp);
    }
    if (nc > (int)(0.9 * A.n) || nc < 1) break;  // coarsening stalled
    HCsr Cc = galerkin(A, agg, nc);
    AmgLevelHost& fine = levels.back();
    fine.nc = nc;
    fine.agg = agg;
    fine.memOff.assign(nc + 1, 0);
    for (int i = 0; i < A.n; ++i) fine.memOff[agg[i] + 1]++;
    for (int I = 0; I < nc; ++I) fine.memOff[I + 1] += fine.memOff[I];
    fine.mem.assign(A.n, 0);
    {
      std::vector<int> fill(fine.memOff.begin(), fine.memOff.end() - 1);
      for (int i = 0; i < A.n; ++i) fine.mem[fill[agg[i]]++] = i;
    }
    AmgLevelHost coarse;
    coarse.n = nc;
    // storage slot of every coarse CSR entry (identity for a CSR level)
    std::vector<int> slot(Cc.off[nc]);
    if (nc > std::max(opt.sellMinRows, 4 * opt.coarseMax)) {
      const int nSl = (nc + kSlice - 1) / kSlice;
      coarse.sliceOff.assign(nSl + 1, 0);
      for (int sl = 0; sl < nSl; ++sl) {
        int w = 0;
        for (int I = sl * kSlice; I < std::min(nc, (sl + 1) * kSlice); ++I) w = std::max(w, Cc.off[I + 1] - Cc.off[I]);
        coarse.maxW = std::max(coarse.maxW, w);
        coarse.sliceOff[sl + 1] = coarse.sliceOff[sl] + w * kSlice;
      }
      coarse.nStore = coarse.sliceOff[nSl];
      coarse.col.assign(coarse.nStore, 0);
      for (int I = 0; I < nc; ++I) {
        const int sl = I / kSlice, lane = I % kSlice;
        const int w = (coarse.sliceOff[sl + 1] - coarse.sliceOff[sl]) / kSlice;
        for (int k = 0; k < w; ++k) {
          const int e = coarse.sliceOff[sl] + k * kSlice + lane;
          const int kk = Cc.off[I] + k;
          if (kk < Cc.off[I + 1]) {
            coarse.col[e] = Cc.col[kk];
            slot[kk] = e;
          } else {
            coarse.col[e] = I;  // padding: the row itself, value 0
          }
        }
      }
    } else {
      coarse.rowOff = Cc.off;
      coarse.col = Cc.col;
      coarse.nStore = Cc.off[nc];
      for (int k = 0; k < Cc.off[nc]; ++k) slot[k] = k;
    }
    // gather lists: coarse storage slots (padding slots get empty lists) then coarse diagonals
    const int nEnt = coarse.nStore;
    std::vector<int> cnt(nEnt + nc + 1, 0);
    std::vector<int> target(A.off[A.n]);
    for (int i = 0; i < A.n; ++i) {
      const int I = agg[i];
      for (int k = A.off[i]; k < A.off[i + 1]; ++k) {
        const int J = agg[A.col[k]];
        int t;
        if (J == I) {
          t = nEnt + I;
        } else {
          const auto b = Cc.col.begin() + Cc.off[I], e = Cc.col.begin() + Cc.off[I + 1];
          t = slot[(int)(std::lower_bound(b, e, J) - Cc.col.begin())];
        }
        target[k] = t;
        cnt[t + 1]++;
      }
      cnt[nEnt + I + 1]++;  // fine diagonal
    }
    fine.gOff.assign(nEnt + nc + 1, 0);
    for (int t = 0; t < nEnt + nc; ++t) fine.gOff[t + 1] = fine.gOff[t] + cnt[t + 1];
    fine.gIdx.assign(fine.gOff.back(), 0);
    {
      std::vector<int> fill(fine.gOff.begin(), fine.gOff.end() - 1);
      for (int i = 0; i < A.n; ++i) {
        for (int k = A.off[i]; k < A.off[i + 1]; ++k) fine.gIdx[fill[target[k]]++] = storage[k];
        fine.gIdx[fill[nEnt + agg[i]]++] = -1 - i;
      }
    }
    levels.push_back(std::move(coarse));
    // storage index of each CSR entry of the new fine level
    A = std::move(Cc);
    storage = std::move(slot);
  }
  return levels;
}

}  // namespace anb
