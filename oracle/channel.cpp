// Oracle-side synthetic channel case: hex mesh generator and boundary-condition evaluation.
// TEST INFRASTRUCTURE ONLY - see oracle.h.  Lets bench.py's reference arm and the CPU tests build
// the benchmark case without the product library.
//
// The generator restates the library's channel mesh (same node coordinates bit for bit, same
// face order), emitting faces directly in their final order instead of sorting them:
//   - internal faces ordered by (owner, neighbour): per cell in id order its +x, +y, +z faces;
//   - boundary faces grouped by patch, then by owner cell, then in the order low-x, high-x,
//     low-y, high-y, low-z, high-z;
//   - nodes not used by any face (inside the removed obstacle) dropped, the rest renumbered in
//     their original order.
// The boundary-condition evaluation restates apply_bc_specs_to_legacy_face_arrays
// (apps/generic_simple_v1/src/velocity_bc_eval.cu:197-290) with the patch geometry table
// (patch_geometry.cu:84-140) for the velocity kinds the channel cases use.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "oracle.h"

namespace {

using V3 = std::array<double, 3>;

struct ChannelTopo {
  std::vector<double> points;
  std::vector<int> faceOff, facePts, owner, neigh, patchStart, patchSize;
};

ChannelTopo make_channel(int nx, int ny, int nz, double Lx, double Ly, double Lz, double jitter, unsigned long long seed,
                         int obstacle, const double box[4]) {
  if (nx < 1 || ny < 1 || nz < 1) throw std::runtime_error("channel mesh needs nx, ny, nz >= 1");
  const double dx = Lx / nx, dy = Ly / ny, dz = Lz / nz;
  // obstacle: the cell-index ranges whose unjittered centres lie in the block
  int i0 = nx, i1 = -1, j0 = ny, j1 = -1;
  if (obstacle) {
    for (int i = 0; i < nx; ++i) {
      const double xc = (i + 0.5) * dx;
      if (xc >= box[0] && xc <= box[1]) i0 = std::min(i0, i), i1 = std::max(i1, i + 1);
    }
    for (int j = 0; j < ny; ++j) {
      const double yc = (j + 0.5) * dy;
      if (yc >= box[2] && yc <= box[3]) j0 = std::min(j0, j), j1 = std::max(j1, j + 1);
    }
    if (i1 <= i0 || j1 <= j0) throw std::runtime_error("obstacle block contains no cell centre");
  }
  const int NX = nx + 1, NY = ny + 1, NZ = nz + 1;
  auto node = [&](int i, int j, int k) { return (k * NY + j) * NX + i; };
  // node coordinates; uniform jitter in [-1, 1) x spacing, three draws per node (x, y, z) in
  // node order; nodes on the box faces and on the obstacle's faces move only tangentially
  std::vector<V3> X((size_t)NX * NY * NZ);
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        const double rx = U(rng);
        const double ry = U(rng);
        const double rz = U(rng);
        bool keepX = i == 0 || i == nx, keepY = j == 0 || j == ny;
        const bool keepZ = k == 0 || k == nz;
        if (obstacle) {
          keepX = keepX || ((i == i0 || i == i1) && j >= j0 && j <= j1);
          keepY = keepY || ((j == j0 || j == j1) && i >= i0 && i <= i1);
        }
        V3 p{i == nx ? Lx : i * dx, j == ny ? Ly : j * dy, k == nz ? Lz : k * dz};
        if (jitter > 0.0) {
          if (!keepX) p[0] += jitter * dx * rx;
          if (!keepY) p[1] += jitter * dy * ry;
          if (!keepZ) p[2] += jitter * dz * rz;
        }
        X[node(i, j, k)] = p;
      }
  // cells in (k, j, i) order without the obstacle block
  std::vector<int> id((size_t)nx * ny * nz, -1);
  std::vector<std::array<int, 3>> ijk;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (obstacle && i >= i0 && i < i1 && j >= j0 && j < j1) continue;
        id[((size_t)k * ny + j) * nx + i] = (int)ijk.size();
        ijk.push_back({i, j, k});
      }
  const int nC = (int)ijk.size();
  // cell across face `side` (0 low, 1 high) of `axis`: id, -1 solid, -2 outside the box
  auto across = [&](const std::array<int, 3>& c, int axis, int side) {
    std::array<int, 3> q = c;
    q[axis] += side ? 1 : -1;
    if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] >= nx || q[1] >= ny || q[2] >= nz) return -2;
    return id[((size_t)q[2] * ny + q[1]) * nx + q[0]];
  };
  // quad on node plane `pl` of `axis` at the cell's other two indices, normal along +axis
  auto quad = [&](const std::array<int, 3>& c, int axis, int pl, int v[4]) {
    const int i = axis == 0 ? pl : c[0], j = axis == 1 ? pl : c[1], k = axis == 2 ? pl : c[2];
    if (axis == 0) {
      v[0] = node(i, j, k); v[1] = node(i, j + 1, k); v[2] = node(i, j + 1, k + 1); v[3] = node(i, j, k + 1);
    } else if (axis == 1) {
      v[0] = node(i, j, k); v[1] = node(i, j, k + 1); v[2] = node(i + 1, j, k + 1); v[3] = node(i + 1, j, k);
    } else {
      v[0] = node(i, j, k); v[1] = node(i + 1, j, k); v[2] = node(i + 1, j + 1, k); v[3] = node(i, j + 1, k);
    }
  };
  ChannelTopo t;
  t.faceOff.push_back(0);
  auto emit = [&](const int v[4], bool reversed) {
    for (int q = 0; q < 4; ++q) t.facePts.push_back(reversed ? v[3 - q] : v[q]);
    t.faceOff.push_back((int)t.facePts.size());
  };
  for (int c = 0; c < nC; ++c)
    for (int axis = 0; axis < 3; ++axis) {
      const int nb = across(ijk[c], axis, 1);
      if (nb < 0) continue;
      int v[4];
      quad(ijk[c], axis, ijk[c][axis] + 1, v);
      emit(v, false);
      t.owner.push_back(c);
      t.neigh.push_back(nb);
    }
  const int nPatch = obstacle ? 4 : 3;
  for (int patch = 0; patch < nPatch; ++patch) {
    t.patchStart.push_back((int)t.owner.size());
    for (int c = 0; c < nC; ++c)
      for (int axis = 0; axis < 3; ++axis)
        for (int side = 0; side < 2; ++side) {
          const int nb = across(ijk[c], axis, side);
          if (nb >= 0) continue;
          const int fp = nb == -1 ? 3 : axis != 0 ? 0 : side == 0 ? 1 : 2;
          if (fp != patch) continue;
          int v[4];
          quad(ijk[c], axis, ijk[c][axis] + side, v);
          emit(v, side == 0);  // the outward normal is -axis on the low side
          t.owner.push_back(c);
        }
    t.patchSize.push_back((int)t.owner.size() - t.patchStart.back());
  }
  // drop the nodes no face uses, keep the others in order
  std::vector<int> newId(X.size(), -1);
  for (int v : t.facePts) newId[v] = 0;
  int nP = 0;
  for (size_t v = 0; v < X.size(); ++v)
    if (newId[v] == 0) {
      newId[v] = nP++;
      for (int q = 0; q < 3; ++q) t.points.push_back(X[v][q]);
    }
  for (int& v : t.facePts) v = newId[v];
  return t;
}

inline double dot3(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// normalize3 of patch_geometry.cu (zero vector below 1e-30)
V3 normalize_or_zero(const V3& a) {
  const double n = std::sqrt(dot3(a, a));
  if (n <= 1.0e-30) return {0.0, 0.0, 0.0};
  return {a[0] / n, a[1] / n, a[2] / n};
}

// normalized_or_throw of velocity_bc_eval.cu:20-28
V3 normalize_or_fail(const V3& a) {
  const double n = std::sqrt(std::max(dot3(a, a), 0.0));
  if (n <= 1.0e-30) throw std::runtime_error("Cannot normalize vector");
  return {a[0] / n, a[1] / n, a[2] / n};
}

}  // namespace

extern "C" {

orc_mesh* orc_channel_create(int nx, int ny, int nz, double Lx, double Ly, double Lz, double jitter,
                             unsigned long long seed, int obstacle, const double* box, char* err, int errlen) {
  try {
    const double defBox[4] = {0.45, 0.55, 0.15, 0.25};
    ChannelTopo t = make_channel(nx, ny, nz, Lx, Ly, Lz, jitter, seed, obstacle, box ? box : defBox);
    const int nF = (int)t.faceOff.size() - 1;
    return orc_mesh_create((int)t.points.size() / 3, t.points.data(), nF, t.faceOff.data(), t.facePts.data(),
                           (int)t.neigh.size(), t.owner.data(), t.neigh.data(), (int)t.patchStart.size(),
                           t.patchStart.data(), t.patchSize.data(), err, errlen);
  } catch (const std::exception& e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return nullptr;
  }
}

int orc_eval_bc(const orc_mesh* m, const int* vkind, const double* vpar, const int* pkind, const double* pval, int* tu,
                int* tv, int* tw, int* tp, double* uf, double* vf, double* wf, double* pf, char* err, int errlen) {
  try {
    int s[6];
    orc_mesh_sizes(m, s);
    const int nF = s[1], nPatch = s[4];
    std::vector<double> xf(3 * (size_t)nF), nf(3 * (size_t)nF), sf(3 * (size_t)nF), af(nF);
    orc_mesh_geometry(m, nullptr, nullptr, xf.data(), nf.data(), sf.data(), af.data(), nullptr);
    std::vector<int> ps(nPatch), pn(nPatch);
    orc_mesh_patches(m, ps.data(), pn.data());
    for (int p = 0; p < nPatch; ++p) {
      const int f0 = ps[p], f1 = ps[p] + pn[p];
      const double* par = vpar + 4 * (size_t)p;
      switch (vkind[p]) {
        case ORC_VEL_ZERO_GRADIENT:
          tu[p] = tv[p] = tw[p] = 0;
          break;
        case ORC_VEL_WALL_NOSLIP:
        case ORC_VEL_UNIFORM:
          tu[p] = tv[p] = tw[p] = 1;
          for (int f = f0; f < f1; ++f) {
            const bool wall = vkind[p] == ORC_VEL_WALL_NOSLIP;
            uf[f] = wall ? 0.0 : par[0];
            vf[f] = wall ? 0.0 : par[1];
            wf[f] = wall ? 0.0 : par[2];
          }
          break;
        case ORC_VEL_PARABOLIC_BOX: {
          // eval_parabolic_box_inlet (velocity_bc_eval.cu:68-100) with AveragePatchNormal: the patch
          // normal is normalize3(sum of Sf in face order) normalised once more, the velocity points
          // inward
          tu[p] = tv[p] = tw[p] = 1;
          const double H = par[0], Umax = par[1];
          const int ia = (int)par[2], ib = (int)par[3];
          if (H <= 0.0 || ia < 0 || ia > 2 || ib < 0 || ib > 2 || ia == ib)
            throw std::runtime_error("invalid parabolic_box_inlet parameters");
          V3 sum{0.0, 0.0, 0.0};
          for (int f = f0; f < f1; ++f)
            for (int q = 0; q < 3; ++q) sum[q] = sum[q] + sf[3 * (size_t)f + q];
          const V3 n = normalize_or_fail(normalize_or_zero(sum));
          const double H2 = H * H, H4 = H2 * H2;
          for (int f = f0; f < f1; ++f) {
            const double a = std::min(std::max(xf[3 * (size_t)f + ia], 0.0), H);
            const double b = std::min(std::max(xf[3 * (size_t)f + ib], 0.0), H);
            const double mag = 16.0 * Umax * a * b * (H - a) * (H - b) / H4;
            uf[f] = -mag * n[0];
            vf[f] = -mag * n[1];
            wf[f] = -mag * n[2];
          }
          break;
        }
        default:
          throw std::runtime_error("unknown velocity kind for patch " + std::to_string(p));
      }
      if (pkind[p] == ORC_P_FIXED_VALUE) {
        tp[p] = 1;
        for (int f = f0; f < f1; ++f) pf[f] = pval[p];
      } else {
        tp[p] = 0;
      }
    }
    return 0;
  } catch (const std::exception& e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
}

}  // extern "C"
