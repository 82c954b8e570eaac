// CPU check of the cluster-resident AMG tail (k_amg_tail_smem in anabasis_b200/csrc/kernels_krylov.cu),
// no GPU needed.
//
// Builds the aggregation hierarchy of a random symmetric M-matrix on an NX x NY x NZ 7-point grid
// (anabasis_b200/csrc/amg_setup.cpp), plans the tail's shared-memory layout with the product's
// planner (plan_smem_tail_layout) and then replays the kernel on the CPU: every CTA's shared memory
// is a byte buffer of the planned size, the staging copies and every later access go through
// bounds-checked helpers, and each read of another CTA's vector entry checks that the owning CTA
// exists and has staged that row.  The tail's result (x2 of its first level) must equal, bit for
// bit, the same V-cycle tail computed on whole-level arrays in the order of resid_csr_rows,
// restrict_rows, dense_rows and up_csr_rows (8 lanes per row, partial sums combined as the
// shuffle tree does).  Prints the plan and "OK"; exits non-zero on the first failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "amg_setup.hpp"

using namespace anb;

namespace {

constexpr int G = 8;  // lanes per row, as kCoarseLanes

int fail(const char* what) {
  std::printf("FAIL: %s\n", what);
  std::exit(1);
}

// sum of the G lanes' partial sums in the order of the shuffle-down tree (offsets 4, 2, 1)
double group_sum(const double (&p)[G]) {
  double v[G];
  for (int i = 0; i < G; ++i) v[i] = p[i];
  for (int o = G / 2; o > 0; o >>= 1)
    for (int i = 0; i < o; ++i) v[i] = v[i] + v[i + o];
  return v[0];
}

// the 32 lanes of a warp summed as warp_sum does (offsets 16 .. 1)
double warp_sum(const double (&p)[32]) {
  double v[32];
  for (int i = 0; i < 32; ++i) v[i] = p[i];
  for (int o = 16; o > 0; o >>= 1)
    for (int i = 0; i < o; ++i) v[i] = v[i] + v[i + o];
  return v[0];
}

struct Cta {  // one CTA's shared memory with bounds-checked typed access
  std::vector<unsigned char> mem;
  std::vector<unsigned char> written;  // byte-level "staged or computed" marks
  template <class T>
  T& at(int off, int idx, int cap) {
    if (idx < 0 || idx >= cap) fail("shared-memory index past its array's capacity");
    const size_t b = (size_t)off + sizeof(T) * (size_t)idx;
    if (b + sizeof(T) > mem.size()) fail("shared-memory access past the planned size");
    return *reinterpret_cast<T*>(&mem[b]);
  }
  template <class T>
  void put(int off, int idx, int cap, T v) {
    at<T>(off, idx, cap) = v;
    const size_t b = (size_t)off + sizeof(T) * (size_t)idx;
    std::memset(&written[b], 1, sizeof(T));
  }
  template <class T>
  T get(int off, int idx, int cap) {
    T v = at<T>(off, idx, cap);
    const size_t b = (size_t)off + sizeof(T) * (size_t)idx;
    for (size_t k = 0; k < sizeof(T); ++k)
      if (!written[b + k]) fail("read of a shared-memory entry that was never written");
    return v;
  }
};

}  // namespace

int main(int argc, char** argv) {
  const int NX = argc > 1 ? std::atoi(argv[1]) : 120, NY = argc > 2 ? std::atoi(argv[2]) : 60,
            NZ = argc > 3 ? std::atoi(argv[3]) : 40, cluster = argc > 4 ? std::atoi(argv[4]) : 16;
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
  Layout Lm;
  Lm.nCells = C;
  Lm.nSlices = (C + kSlice - 1) / kSlice;
  Lm.rowLen.resize(C);
  Lm.sliceOff.assign(Lm.nSlices + 1, 0);
  for (int r = 0; r < C; ++r) Lm.rowLen[r] = (int)nb[r].size();
  for (int s = 0; s < Lm.nSlices; ++s) {
    int w = 0;
    for (int r = s * kSlice; r < std::min(C, (s + 1) * kSlice); ++r) w = std::max(w, Lm.rowLen[r]);
    Lm.maxRowLen = std::max(Lm.maxRowLen, w);
    Lm.sliceOff[s + 1] = Lm.sliceOff[s] + w * kSlice;
  }
  auto slot = [&](int r, int k) { return Lm.sliceOff[r / kSlice] + kSlice * k + r % kSlice; };
  Lm.col.assign(Lm.sliceOff.back(), 0);
  std::vector<double> val0(Lm.sliceOff.back(), 0.0), diag0(C, 0.1);
  for (int r = 0; r < C; ++r)
    for (int k = 0; k < (Lm.sliceOff[r / kSlice + 1] - Lm.sliceOff[r / kSlice]) / kSlice; ++k)
      Lm.col[slot(r, k)] = k < Lm.rowLen[r] ? nb[r][k] : r;
  std::mt19937 g(11);
  std::uniform_real_distribution<double> U(0.5, 1.5);
  for (int r = 0; r < C; ++r)
    for (int k = 0; k < Lm.rowLen[r]; ++k) {
      const int c = nb[r][k];
      if (c < r) continue;
      const double a = -U(g);
      val0[slot(r, k)] = a;
      for (int k2 = 0; k2 < Lm.rowLen[c]; ++k2)
        if (nb[c][k2] == r) val0[slot(c, k2)] = a;
      diag0[r] -= a;
      diag0[c] -= a;
    }
  AmgSetupOptions opt;
  const auto H = build_amg_hierarchy(Lm, val0, diag0, opt);
  const int L = (int)H.size();
  // coarse values through the Galerkin gather lists (as k_amg_galerkin), smoother weights 0.9 / d
  std::vector<std::vector<double>> val(L), diag(L), wd(L);
  val[0] = val0;
  diag[0] = diag0;
  for (int l = 0; l + 1 < L; ++l) {
    const AmgLevelHost& f = H[l];
    const AmgLevelHost& c = H[l + 1];
    val[l + 1].assign(c.nStore, 0.0);
    diag[l + 1].assign(c.n, 0.0);
    for (int t = 0; t < c.nStore + c.n; ++t) {
      double s = 0.0;
      for (int k = f.gOff[t]; k < f.gOff[t + 1]; ++k) {
        const int idx = f.gIdx[k];
        s += idx >= 0 ? val[l][idx] : diag[l][-1 - idx];
      }
      (t < c.nStore ? val[l + 1][t] : diag[l + 1][t - c.nStore]) = s;
    }
  }
  for (int l = 0; l < L; ++l) {
    wd[l].resize(H[l].n);
    for (int i = 0; i < H[l].n; ++i) wd[l][i] = 0.9 / diag[l][i];
  }

  std::vector<SmemTailLevel> lay(L);
  size_t bytes = 0;
  const int t0 = plan_smem_tail_layout(H, cluster, sizeof(double), 227 * 1024, 12, lay.data(), &bytes);
  std::printf("levels:");
  for (int l = 0; l < L; ++l) std::printf(" %d%s", H[l].n, H[l].sliceOff.empty() ? "" : "(SELL)");
  std::printf("\ntail from level %d on %d CTAs, %zu bytes of shared memory each\n", t0, cluster, bytes);
  if (t0 == 0) fail("no level fits");
  const int nD = H[L - 1].n;
  std::vector<double> inv((size_t)nD * nD);
  for (double& v : inv) v = U(g) - 1.0;
  const double corr = 1.6;
  std::vector<double> b0(H[t0].n);
  for (double& v : b0) v = U(g) - 1.0;

  // reference: whole-level arrays, the L2-based tail's order
  std::vector<std::vector<double>> rb(L), rx(L), rx2(L);
  for (int l = t0; l < L; ++l) rb[l].assign(H[l].n, 0.0), rx[l].assign(H[l].n, 0.0), rx2[l].assign(H[l].n, 0.0);
  rb[t0] = b0;
  for (int l = t0; l + 1 < L; ++l) {
    const AmgLevelHost& f = H[l];
    for (int i = 0; i < f.n; ++i) {
      double p[G] = {};
      for (int s = 0; s < G; ++s)
        for (int k = f.rowOff[i] + s; k < f.rowOff[i + 1]; k += G) {
          const int j = f.col[k];
          p[s] += val[l][k] * (wd[l][j] * rb[l][j]);
        }
      const double acc = group_sum(p), xi = wd[l][i] * rb[l][i];
      rx[l][i] = xi;
      rx2[l][i] = rb[l][i] - diag[l][i] * xi - acc;
    }
    for (int I = 0; I < f.nc; ++I) {
      double acc = 0.0;
      for (int m = f.memOff[I]; m < f.memOff[I + 1]; ++m) acc += rx2[l][f.mem[m]];
      rb[l + 1][I] = acc;
    }
  }
  for (int i = 0; i < nD; ++i) {
    double p[32] = {};
    for (int s = 0; s < 32; ++s)
      for (int j = s; j < nD; j += 32) p[s] += inv[(size_t)i * nD + j] * rb[L - 1][j];
    rx[L - 1][i] = warp_sum(p);
  }
  for (int l = L - 2; l >= t0; --l) {
    const AmgLevelHost& f = H[l];
    const std::vector<double>& e = (l + 1 == L - 1) ? rx[l + 1] : rx2[l + 1];
    std::vector<double> out(f.n);
    for (int i = 0; i < f.n; ++i) {
      double p[G] = {};
      for (int s = 0; s < G; ++s)
        for (int k = f.rowOff[i] + s; k < f.rowOff[i + 1]; k += G) {
          const int j = f.col[k];
          p[s] += val[l][k] * (rx[l][j] + corr * e[f.agg[j]]);
        }
      const double acc = group_sum(p);
      const double xi = rx[l][i] + corr * e[f.agg[i]];
      out[i] = xi + wd[l][i] * (rb[l][i] - diag[l][i] * xi - acc);
    }
    rx2[l] = out;
  }

  // replay of k_amg_tail_smem: staging, then the sweeps phase by phase over all CTAs
  std::vector<Cta> cta(cluster);
  for (Cta& c : cta) c.mem.assign(bytes, 0), c.written.assign(bytes, 0);
  auto own = [&](int l, int r, int& r0, int& nl) {
    r0 = std::min(H[l].n, r * lay[l].cs);
    nl = std::min(H[l].n, r0 + lay[l].cs) - r0;
  };
  auto dsm = [&](int l, int off, int j) {  // another CTA's entry j of a level-l vector at offset off
    if (j < 0 || j >= H[l].n) fail("vector index out of the level");
    const int cs = lay[l].cs, r = j / cs;
    if (r >= cluster) fail("owning CTA past the cluster");
    return cta[r].get<double>(off, j - r * cs, cs);
  };
  auto capE = [&](int l) { return (lay[l].oCol - lay[l].oVal) / (int)sizeof(double); };
  auto capM = [&](int l) { return (lay[l + 1].oB - lay[l].oMem) / 2; };
  for (int r = 0; r < cluster; ++r) {
    Cta& c = cta[r];
    for (int l = t0; l < L; ++l) {
      const AmgLevelHost& f = H[l];
      const SmemTailLevel& s = lay[l];
      int r0, nl;
      own(l, r, r0, nl);
      if (l == t0)
        for (int i = 0; i < nl; ++i) c.put<double>(s.oB, i, s.cs, b0[r0 + i]);
      if (l + 1 == L) break;
      const int e0 = f.rowOff[r0], ne = f.rowOff[r0 + nl] - e0;
      for (int k = 0; k < ne; ++k) {
        c.put<double>(s.oVal, k, capE(l), val[l][e0 + k]);
        c.put<unsigned short>(s.oCol, k, capE(l), (unsigned short)f.col[e0 + k]);
        c.put<unsigned short>(s.oColAgg, k, capE(l), (unsigned short)f.agg[f.col[e0 + k]]);
      }
      for (int i = 0; i <= nl; ++i) {
        c.put<int>(s.oRow, i, s.cs + 1, f.rowOff[r0 + i] - e0);
        if (i < nl) {
          c.put<double>(s.oDiag, i, s.cs, diag[l][r0 + i]);
          c.put<double>(s.oWd, i, s.cs, wd[l][r0 + i]);
          c.put<unsigned short>(s.oAgg, i, s.cs, (unsigned short)f.agg[r0 + i]);
        }
      }
      const SmemTailLevel& sn = lay[l + 1];
      int I0, nI;
      own(l + 1, r, I0, nI);
      const int m0 = f.memOff[I0], nm = f.memOff[I0 + nI] - m0;
      for (int I = 0; I <= nI; ++I) c.put<int>(s.oMemOff, I, sn.cs + 1, f.memOff[I0 + I] - m0);
      for (int m = 0; m < nm; ++m) c.put<unsigned short>(s.oMem, m, capM(l), (unsigned short)f.mem[m0 + m]);
    }
  }
  for (int l = t0; l + 1 < L; ++l) {
    const SmemTailLevel& s = lay[l];
    for (int r = 0; r < cluster; ++r) {
      Cta& c = cta[r];
      int r0, nl;
      own(l, r, r0, nl);
      for (int i = 0; i < nl; ++i) {
        double p[G] = {};
        const int k1 = c.get<int>(s.oRow, i + 1, s.cs + 1);
        for (int sub = 0; sub < G; ++sub)
          for (int k = c.get<int>(s.oRow, i, s.cs + 1) + sub; k < k1; k += G) {
            const int j = c.get<unsigned short>(s.oCol, k, capE(l));
            p[sub] += c.get<double>(s.oVal, k, capE(l)) * (dsm(l, s.oWd, j) * dsm(l, s.oB, j));
          }
        const double acc = group_sum(p), bi = c.get<double>(s.oB, i, s.cs);
        const double xi = c.get<double>(s.oWd, i, s.cs) * bi;
        c.put<double>(s.oX, i, s.cs, xi);
        c.put<double>(s.oX2, i, s.cs, bi - c.get<double>(s.oDiag, i, s.cs) * xi - acc);
      }
    }
    const SmemTailLevel& sn = lay[l + 1];
    for (int r = 0; r < cluster; ++r) {
      Cta& c = cta[r];
      int I0, nI;
      own(l + 1, r, I0, nI);
      for (int I = 0; I < nI; ++I) {
        double acc = 0.0;
        const int m1 = c.get<int>(s.oMemOff, I + 1, sn.cs + 1);
        for (int m = c.get<int>(s.oMemOff, I, sn.cs + 1); m < m1; ++m)
          acc += dsm(l, s.oX2, c.get<unsigned short>(s.oMem, m, capM(l)));
        c.put<double>(sn.oB, I, sn.cs, acc);
      }
    }
  }
  {
    const SmemTailLevel& s = lay[L - 1];
    for (int r = 0; r < cluster; ++r) {
      int r0, nl;
      own(L - 1, r, r0, nl);
      for (int i = 0; i < nl; ++i) {
        double p[32] = {};
        for (int sub = 0; sub < 32; ++sub)
          for (int j = sub; j < nD; j += 32) p[sub] += inv[(size_t)(r0 + i) * nD + j] * dsm(L - 1, s.oB, j);
        cta[r].put<double>(s.oX, i, s.cs, warp_sum(p));
      }
    }
  }
  std::vector<double> got(H[t0].n, NAN);
  for (int l = L - 2; l >= t0; --l) {
    const SmemTailLevel& s = lay[l];
    const SmemTailLevel& sn = lay[l + 1];
    const int eoff = (l + 1 == L - 1) ? sn.oX : sn.oX2;
    std::vector<std::vector<double>> outs(cluster);
    for (int r = 0; r < cluster; ++r) {
      Cta& c = cta[r];
      int r0, nl;
      own(l, r, r0, nl);
      outs[r].resize(nl);
      for (int i = 0; i < nl; ++i) {
        double p[G] = {};
        const int k1 = c.get<int>(s.oRow, i + 1, s.cs + 1);
        for (int sub = 0; sub < G; ++sub)
          for (int k = c.get<int>(s.oRow, i, s.cs + 1) + sub; k < k1; k += G)
            p[sub] += c.get<double>(s.oVal, k, capE(l)) *
                      (dsm(l, s.oX, c.get<unsigned short>(s.oCol, k, capE(l))) +
                       corr * dsm(l + 1, eoff, c.get<unsigned short>(s.oColAgg, k, capE(l))));
        const double acc = group_sum(p);
        const double xi = c.get<double>(s.oX, i, s.cs) + corr * dsm(l + 1, eoff, c.get<unsigned short>(s.oAgg, i, s.cs));
        outs[r][i] = xi + c.get<double>(s.oWd, i, s.cs) *
                              (c.get<double>(s.oB, i, s.cs) - c.get<double>(s.oDiag, i, s.cs) * xi - acc);
      }
    }
    for (int r = 0; r < cluster; ++r) {  // written after every CTA's reads of this phase
      int r0, nl;
      own(l, r, r0, nl);
      for (int i = 0; i < nl; ++i) {
        if (l == t0) got[r0 + i] = outs[r][i];
        else cta[r].put<double>(s.oX2, i, s.cs, outs[r][i]);
      }
    }
  }
  for (int i = 0; i < H[t0].n; ++i)
    if (!(got[i] == rx2[t0][i])) fail("tail result differs from the whole-level computation");
  std::printf("OK\n");
  return 0;
}
