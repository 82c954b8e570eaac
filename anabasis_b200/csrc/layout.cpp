// Device layout builder: RCM renumbering, SELL-32 pattern, face coefficients, LSQ moments.
#include "layout.hpp"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <numeric>
#include <queue>
#include <stdexcept>

namespace anb {

// Reverse Cuthill-McKee order of the cell graph: per connected component, a pseudo-peripheral
// start (up to four BFS sweeps, each restarted from the last level's lowest-degree node), then a
// BFS that appends each node's unvisited neighbours by ascending (degree, index); the whole order
// reversed.  Queues are flat arrays (the order itself for the final BFS).
std::vector<int> rcm_order(int n, const std::vector<int>& off, const std::vector<int>& adj) {
  std::vector<int> deg(n);
  for (int i = 0; i < n; ++i) deg[i] = off[i + 1] - off[i];
  std::vector<int> order;
  order.reserve(n);
  std::vector<char> seen(n, 0);
  std::vector<int> level(n, -1);
  std::vector<int> q;
  q.reserve(n);
  // BFS from s; returns the lowest-degree node (first met) of the last level, depth = its level
  auto bfs_last = [&](int s, int& depth) {
    q.clear();
    q.push_back(s);
    level[s] = 0;
    int last = s;
    depth = 0;
    for (size_t h = 0; h < q.size(); ++h) {
      const int v = q[h];
      if (level[v] > depth || (level[v] == depth && deg[v] < deg[last])) {
        depth = level[v];
        last = v;
      }
      for (int k = off[v]; k < off[v + 1]; ++k) {
        const int w = adj[k];
        if (level[w] < 0) {
          level[w] = level[v] + 1;
          q.push_back(w);
        }
      }
    }
    for (int v : q) level[v] = -1;
    return last;
  };
  std::vector<int> nb;
  for (int s0 = 0; s0 < n; ++s0) {
    if (seen[s0]) continue;
    int s = s0, d0 = -1;
    for (int it = 0; it < 4; ++it) {
      int d;
      const int t = bfs_last(s, d);
      if (d <= d0) break;
      d0 = d;
      s = t;
    }
    size_t h = order.size();
    order.push_back(s);
    seen[s] = 1;
    while (h < order.size()) {
      const int v = order[h++];
      nb.clear();
      for (int k = off[v]; k < off[v + 1]; ++k)
        if (!seen[adj[k]]) nb.push_back(adj[k]);
      // insertion sort by (degree, index): the lists are a handful of entries
      for (size_t i = 1; i < nb.size(); ++i) {
        const int x = nb[i];
        size_t j = i;
        while (j > 0 && (deg[nb[j - 1]] > deg[x] || (deg[nb[j - 1]] == deg[x] && nb[j - 1] > x))) {
          nb[j] = nb[j - 1];
          --j;
        }
        nb[j] = x;
      }
      for (int w : nb) {
        seen[w] = 1;
        order.push_back(w);
      }
    }
  }
  std::reverse(order.begin(), order.end());
  return order;
}

void cell_adjacency(const HostMesh& m, std::vector<int>& off, std::vector<int>& adj) {
  const int C = m.nCells, nI = m.nInternalFaces;
  off.assign(C + 1, 0);
  std::vector<int> cnt(C + 1, 0);
  for (int f = 0; f < nI; ++f) {
    cnt[m.owner[f] + 1]++;
    cnt[m.neigh[f] + 1]++;
  }
  for (int c = 0; c < C; ++c) off[c + 1] = off[c] + cnt[c + 1];
  adj.assign(off[C], 0);
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (int f = 0; f < nI; ++f) {
    adj[fill[m.owner[f]]++] = m.neigh[f];
    adj[fill[m.neigh[f]]++] = m.owner[f];
  }
  int dup = -1;
#pragma omp parallel for schedule(static) reduction(max : dup)
  for (int c = 0; c < C; ++c) {
    auto b = adj.begin() + off[c], e = adj.begin() + off[c + 1];
    std::sort(b, e);
    if (std::adjacent_find(b, e) != e) dup = std::max(dup, C - 1 - c);  // keep the lowest such cell
  }
  if (dup >= 0)
    throw std::runtime_error("cell " + std::to_string(C - 1 - dup) +
                             " shares more than one internal face with a neighbour (unsupported)");
}

std::vector<double> lsq_minv_host(const HostMesh& m, const std::vector<int>& off, const std::vector<int>& adj) {
  const int C = m.nCells, nI = m.nInternalFaces, nF = m.nFaces;
  std::vector<double> minvOrig((size_t)6 * C, 0.0);
  std::vector<std::vector<int>> cellB(C);
  for (int f = nI; f < nF; ++f) cellB[m.owner[f]].push_back(f);
#pragma omp parallel for schedule(static)
  for (int P = 0; P < C; ++P) {
    const Vec3 xP = m.cc[P];
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    auto acc = [&](const Vec3& x) {
      double r[3] = {x[0] - xP[0], x[1] - xP[1], x[2] - xP[2]};
      double w = 1.0 / std::max(r[0] * r[0] + r[1] * r[1] + r[2] * r[2], 1e-30);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i][j] += w * r[i] * r[j];
    };
    for (int k = off[P]; k < off[P + 1]; ++k) acc(m.cc[adj[k]]);
    for (int f : cellB[P]) acc(m.xf[f]);
    double a = M[0][0], b = M[0][1], c = M[0][2], d = M[1][0], e = M[1][1], f2 = M[1][2], g = M[2][0],
           h = M[2][1], k = M[2][2];
    double det = a * (e * k - f2 * h) - b * (d * k - f2 * g) + c * (d * h - e * g);
    double* o = &minvOrig[(size_t)6 * P];
    if (std::fabs(det) > 1e-20) {
      o[0] = (e * k - f2 * h) / det;
      o[1] = (c * h - b * k) / det;
      o[2] = (b * f2 - c * e) / det;
      o[3] = (a * k - c * g) / det;
      o[4] = (c * d - a * f2) / det;
      o[5] = (a * e - b * d) / det;
    }
  }
  return minvOrig;
}

Layout build_layout(const HostMesh& m) {
  std::vector<int> off, adj;
  cell_adjacency(m, off, adj);
  const std::vector<double> minv = lsq_minv_host(m, off, adj);
  return build_layout(m, off, adj, minv);
}

Layout build_layout(const HostMesh& m, const std::vector<int>& off, const std::vector<int>& adj,
                    const std::vector<double>& minvOrig) {
  Layout L;
  const int C = m.nCells, nI = m.nInternalFaces, nF = m.nFaces;
  L.nCells = C;
  L.nInternal = nI;
  L.nBoundary = nF - nI;
  L.nPatches = (int)m.patches.size();
  auto clk = std::chrono::steady_clock::now();
  auto lap = [&](int k) {
    const auto t = std::chrono::steady_clock::now();
    L.seconds[k] = std::chrono::duration<double>(t - clk).count();
    clk = t;
  };
  lap(0);
  lap(1);
  // RCM renumbering
  L.new2old = rcm_order(C, off, adj);
  L.old2new.assign(C, 0);
  for (int i = 0; i < C; ++i) L.old2new[L.new2old[i]] = i;
  lap(2);

  // internal faces re-oriented (owner < neighbour in new ids) and ordered by (owner, neighbour):
  // counted into owner buckets, each bucket sorted by neighbour (pairs are distinct)
  std::vector<int> fperm(nI);
  {
    std::vector<int> lo(nI), hi(nI), bOff(C + 1, 0);
#pragma omp parallel for schedule(static)
    for (int f = 0; f < nI; ++f) {
      const int a = L.old2new[m.owner[f]], b = L.old2new[m.neigh[f]];
      lo[f] = std::min(a, b);
      hi[f] = std::max(a, b);
    }
    for (int f = 0; f < nI; ++f) bOff[lo[f] + 1]++;
    for (int r = 0; r < C; ++r) bOff[r + 1] += bOff[r];
    std::vector<int> fill(bOff.begin(), bOff.end() - 1);
    for (int f = 0; f < nI; ++f) fperm[fill[lo[f]]++] = f;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < C; ++r)
      std::sort(fperm.begin() + bOff[r], fperm.begin() + bOff[r + 1], [&](int x, int y) { return hi[x] < hi[y]; });
  }
  L.fOwner.resize(nI);
  L.fNeigh.resize(nI);
  L.fOrig.resize(nI);
  L.fFlip.resize(nI);
  L.fLam.resize(nI);
  L.fG.resize(nI);
  L.fT.resize((size_t)3 * nI);
  L.fD.resize((size_t)3 * nI);
  L.fFlags.resize(nI);
#pragma omp parallel for schedule(static)
  for (int fi = 0; fi < nI; ++fi) {
    const int f = fperm[fi];
    const int o = L.old2new[m.owner[f]], n = L.old2new[m.neigh[f]];
    const bool flip = o > n;
    const int P = flip ? m.neigh[f] : m.owner[f];  // original ids of the new owner / neighbour
    const int N = flip ? m.owner[f] : m.neigh[f];
    L.fOwner[fi] = std::min(o, n);
    L.fNeigh[fi] = std::max(o, n);
    L.fOrig[fi] = f;
    L.fFlip[fi] = flip ? 1 : 0;
    const double sg = flip ? -1.0 : 1.0;
    const double d[3] = {m.cc[N][0] - m.cc[P][0], m.cc[N][1] - m.cc[P][1], m.cc[N][2] - m.cc[P][2]};
    const double S[3] = {sg * m.Sf[f][0], sg * m.Sf[f][1], sg * m.Sf[f][2]};
    const double nv[3] = {sg * m.nf[f][0], sg * m.nf[f][1], sg * m.nf[f][2]};
    const double nd = nv[0] * d[0] + nv[1] * d[1] + nv[2] * d[2];
    const double den = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double lam = ((m.xf[f][0] - m.cc[P][0]) * d[0] + (m.xf[f][1] - m.cc[P][1]) * d[1] +
                  (m.xf[f][2] - m.cc[P][2]) * d[2]) /
                 (den > 1e-30 ? den : 1e-30);
    lam = std::min(1.0, std::max(0.0, lam));
    const double A = m.Af[f];
    const double g = A / std::max(std::fabs(nd), 1e-30);
    L.fLam[fi] = lam;
    L.fG[fi] = g;
    for (int k = 0; k < 3; ++k) {
      L.fD[(size_t)3 * fi + k] = d[k];
      L.fT[(size_t)3 * fi + k] = S[k] - g * d[k];
    }
    L.fFlags[fi] = (uint8_t)((nd > 1e-14 ? kFaceAsm : 0) | (std::fabs(nd) > 1e-30 ? kFaceNonOrth : 0));
  }

  lap(3);
  // SELL-32 pattern: row r lists its neighbours ascending with the connecting face
  std::vector<int> rOff(C + 1, 0);
  for (int fi = 0; fi < nI; ++fi) {
    rOff[L.fOwner[fi] + 1]++;
    rOff[L.fNeigh[fi] + 1]++;
  }
  for (int r = 0; r < C; ++r) rOff[r + 1] += rOff[r];
  std::vector<int> rCol(rOff[C]), rFace(rOff[C]);
  {
    std::vector<int> fill(rOff.begin(), rOff.end() - 1);
    // neighbours below r come from faces where r is the neighbour; faces are sorted by
    // (owner, neighbour) so a pass over faces yields ascending owners per neighbour row
    for (int fi = 0; fi < nI; ++fi) {
      int n = L.fNeigh[fi];
      rCol[fill[n]] = L.fOwner[fi];
      rFace[fill[n]++] = fi;
    }
    for (int fi = 0; fi < nI; ++fi) {
      int o = L.fOwner[fi];
      rCol[fill[o]] = L.fNeigh[fi];
      rFace[fill[o]++] = fi;
    }
  }
  L.rowLen.resize(C);
  for (int r = 0; r < C; ++r) L.rowLen[r] = rOff[r + 1] - rOff[r];
  L.nSlices = (C + kSlice - 1) / kSlice;
  L.sliceOff.assign(L.nSlices + 1, 0);
  L.maxRowLen = 0;
  for (int s = 0; s < L.nSlices; ++s) {
    int w = 0;
    for (int r = s * kSlice; r < std::min(C, (s + 1) * kSlice); ++r) w = std::max(w, L.rowLen[r]);
    L.maxRowLen = std::max(L.maxRowLen, w);
    L.sliceOff[s + 1] = L.sliceOff[s] + w * kSlice;
  }
  L.col.assign(L.sliceOff[L.nSlices], 0);
  L.slotFace.assign(L.sliceOff[L.nSlices], -1);
#pragma omp parallel for schedule(static)
  for (int s = 0; s < L.nSlices; ++s) {
    const int w = (L.sliceOff[s + 1] - L.sliceOff[s]) / kSlice;
    for (int lane = 0; lane < kSlice; ++lane) {
      const int r = s * kSlice + lane;
      for (int k = 0; k < w; ++k) {
        const size_t e = (size_t)L.sliceOff[s] + (size_t)k * kSlice + lane;
        if (r < C && k < L.rowLen[r]) {
          L.col[e] = rCol[rOff[r] + k];
          L.slotFace[e] = rFace[rOff[r] + k];
        } else {
          L.col[e] = r < C ? r : 0;
          L.slotFace[e] = -1;
        }
      }
    }
  }

  lap(4);
  // boundary faces (input order)
  const int nB = nF - nI;
  L.bOwner.resize(nB);
  L.bPatch.resize(nB);
  L.bG.resize(nB);
  L.bT.resize((size_t)3 * nB);
  L.bS.resize((size_t)3 * nB);
  L.bFlags.resize(nB);
  int noPatch = INT_MAX;
#pragma omp parallel for schedule(static) reduction(min : noPatch)
  for (int b = 0; b < nB; ++b) {
    const int f = nI + b;
    const int P = m.owner[f];
    L.bOwner[b] = L.old2new[P];
    L.bPatch[b] = m.bPatch[f] - 1;
    if (L.bPatch[b] < 0) noPatch = std::min(noPatch, f);
    const double d[3] = {m.xf[f][0] - m.cc[P][0], m.xf[f][1] - m.cc[P][1], m.xf[f][2] - m.cc[P][2]};
    const double nd = m.nf[f][0] * d[0] + m.nf[f][1] * d[1] + m.nf[f][2] * d[2];
    const double g = m.Af[f] / std::max(std::fabs(nd), 1e-30);
    L.bG[b] = g;
    for (int k = 0; k < 3; ++k) {
      L.bS[(size_t)3 * b + k] = m.Sf[f][k];
      L.bT[(size_t)3 * b + k] = m.Sf[f][k] - g * d[k];
    }
    L.bFlags[b] = (uint8_t)((nd > 1e-14 ? kFaceAsm : 0) | (std::fabs(nd) > 1e-30 ? kFaceNonOrth : 0));
  }
  if (noPatch != INT_MAX) throw std::runtime_error("boundary face " + std::to_string(noPatch) + " belongs to no patch");
  L.cbOff.assign(C + 1, 0);
  for (int b = 0; b < nB; ++b) L.cbOff[L.bOwner[b] + 1]++;
  for (int r = 0; r < C; ++r) L.cbOff[r + 1] += L.cbOff[r];
  L.cbList.assign(nB, 0);
  {
    std::vector<int> fill(L.cbOff.begin(), L.cbOff.end() - 1);
    for (int b = 0; b < nB; ++b) L.cbList[fill[L.bOwner[b]]++] = b;
  }

  // cell data in new order
  L.vol.resize(C);
  L.cc.resize((size_t)3 * C);
  L.minv.resize((size_t)6 * C);
#pragma omp parallel for schedule(static)
  for (int r = 0; r < C; ++r) {
    const int o = L.new2old[r];
    L.vol[r] = m.vol[o];
    for (int k = 0; k < 3; ++k) L.cc[(size_t)3 * r + k] = m.cc[o][k];
    for (int k = 0; k < 6; ++k) L.minv[(size_t)6 * r + k] = minvOrig[(size_t)6 * o + k];
  }
  lap(5);
  return L;
}

std::vector<double> scalar_lsq_minv(const HostMesh& m, const Layout& L, const std::vector<uint8_t>& bDirichlet) {
  const int C = m.nCells, nI = m.nInternalFaces, nF = m.nFaces;
  if ((int)bDirichlet.size() != nF - nI) throw std::runtime_error("scalar_lsq_minv: boundary type size mismatch");
  // sorted unique neighbours (cellNbrs) and ascending boundary faces (cellBFace) per cell
  std::vector<int> off(C + 1, 0), adj;
  for (int f = 0; f < nI; ++f) {
    ++off[m.owner[f] + 1];
    ++off[m.neigh[f] + 1];
  }
  for (int c = 0; c < C; ++c) off[c + 1] += off[c];
  adj.resize(off[C]);
  {
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int f = 0; f < nI; ++f) {
      adj[fill[m.owner[f]]++] = m.neigh[f];
      adj[fill[m.neigh[f]]++] = m.owner[f];
    }
  }
  std::vector<std::vector<int>> cellB(C);
  for (int f = nI; f < nF; ++f) cellB[m.owner[f]].push_back(f);
  std::vector<double> out((size_t)6 * C, 0.0);
#pragma omp parallel for schedule(static)
  for (int P = 0; P < C; ++P) {
    std::sort(adj.begin() + off[P], adj.begin() + off[P + 1]);
    const Vec3 xP = m.cc[P];
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    auto acc = [&](const double r[3]) {
      const double w = 1.0 / std::max(r[0] * r[0] + r[1] * r[1] + r[2] * r[2], 1e-30);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i][j] += w * r[i] * r[j];
    };
    for (int k = off[P]; k < off[P + 1]; ++k) {
      const Vec3& x = m.cc[adj[k]];
      const double r[3] = {x[0] - xP[0], x[1] - xP[1], x[2] - xP[2]};
      acc(r);
    }
    for (int f : cellB[P]) {
      const double rcf[3] = {m.xf[f][0] - xP[0], m.xf[f][1] - xP[1], m.xf[f][2] - xP[2]};
      if (bDirichlet[f - nI]) {
        acc(rcf);
      } else {
        const Vec3& n = m.nf[f];
        const double dn = std::max(rcf[0] * n[0] + rcf[1] * n[1] + rcf[2] * n[2], 1e-30);
        const double r[3] = {dn * n[0], dn * n[1], dn * n[2]};
        acc(r);
      }
    }
    const double a = M[0][0], b = M[0][1], c = M[0][2], d = M[1][0], e = M[1][1], f2 = M[1][2], g = M[2][0],
                 h = M[2][1], k = M[2][2];
    const double det = a * (e * k - f2 * h) - b * (d * k - f2 * g) + c * (d * h - e * g);
    double* o = &out[(size_t)6 * L.old2new[P]];
    if (std::fabs(det) > 1e-20) {
      o[0] = (e * k - f2 * h) / det;
      o[1] = (c * h - b * k) / det;
      o[2] = (b * f2 - c * e) / det;
      o[3] = (a * k - c * g) / det;
      o[4] = (c * d - a * f2) / det;
      o[5] = (a * e - b * d) / det;
    }
  }
  return out;
}

}  // namespace anb
