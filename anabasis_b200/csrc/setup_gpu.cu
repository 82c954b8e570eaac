// Mesh set-up on the device: cell and face geometry (read_openfoam_polymesh, main.cu:591-597),
// the least-squares moment inverse (build_lsq_gradient_operator, main.cu:1169-1224) and the
// slot-ordered copy of the face records.
//
// The geometry and moment kernels reproduce the host restatement (host_mesh.cpp compute_geometry,
// layout.cpp) bit for bit, and through it the reference: every sum, product and difference is an
// explicit round-to-nearest intrinsic in the host code's order, so nothing is contracted into a
// fused multiply-add, and division and square root are the correctly rounded IEEE operations.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "setup_gpu.hpp"

namespace anb {
namespace {

constexpr int kMaxCellVerts = 64;  // distinct points of one cell handled on the device

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ D3 add3(D3 a, D3 b) { return {__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y), __dadd_rn(a.z, b.z)}; }
__device__ __forceinline__ D3 sub3(D3 a, D3 b) { return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)}; }
__device__ __forceinline__ D3 mul3(double s, D3 a) { return {__dmul_rn(s, a.x), __dmul_rn(s, a.y), __dmul_rn(s, a.z)}; }
__device__ __forceinline__ double dot3(D3 a, D3 b) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dmul_rn(a.z, b.z));
}
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
  return {__dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)), __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
          __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x))};
}
__device__ __forceinline__ void st3(double* p, D3 v) {
  p[0] = v.x;
  p[1] = v.y;
  p[2] = v.z;
}

// Cell volume and centroid by tetrahedra about the vertex average (compute_geometry): the cell's
// distinct points ascending, their average c0, then per face (neighbour-side faces reversed) the
// fan of tetrahedra (c0, a, b, d) from the face's first point.
__global__ void k_cell_geom(int nC, const int* __restrict__ cfOff, const int* __restrict__ cfFace,
                            const signed char* __restrict__ cfOri, const int* __restrict__ faceOff,
                            const int* __restrict__ facePts, const double* __restrict__ P, double* vol, double* cc,
                            int* badCell, int* overflow) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nC; c += gridDim.x * blockDim.x) {
    int verts[kMaxCellVerts];
    int nv = 0;
    bool over = false;
    for (int j = cfOff[c]; j < cfOff[c + 1] && !over; ++j) {
      const int f = cfFace[j];
      for (int k = faceOff[f]; k < faceOff[f + 1]; ++k) {
        const int v = facePts[k];
        int pos = nv;  // insertion into the ascending list of distinct points
        while (pos > 0 && verts[pos - 1] > v) --pos;
        if (pos > 0 && verts[pos - 1] == v) continue;
        if (nv == kMaxCellVerts) {
          over = true;
          break;
        }
        for (int q = nv; q > pos; --q) verts[q] = verts[q - 1];
        verts[pos] = v;
        ++nv;
      }
    }
    if (over) {
      atomicExch(overflow, 1);
      continue;
    }
    D3 c0{0.0, 0.0, 0.0};
    for (int q = 0; q < nv; ++q) c0 = add3(c0, ld3(P + 3 * (size_t)verts[q]));
    c0 = mul3(1.0 / (double)max(nv, 1), c0);
    double V = 0.0;
    D3 M{0.0, 0.0, 0.0};
    for (int j = cfOff[c]; j < cfOff[c + 1]; ++j) {
      const int f = cfFace[j];
      const int b0 = faceOff[f], n = faceOff[f + 1] - b0;
      const bool rev = cfOri[j] < 0;
      auto pt = [&](int i) { return ld3(P + 3 * (size_t)facePts[b0 + (rev ? n - 1 - i : i)]); };
      const D3 a = pt(0);
      for (int i = 1; i + 1 < n; ++i) {
        const D3 b = pt(i), d = pt(i + 1);
        const double vTet = __ddiv_rn(dot3(sub3(a, c0), cross3(sub3(b, c0), sub3(d, c0))), 6.0);
        const D3 cTet = mul3(0.25, add3(add3(c0, a), add3(b, d)));
        V = __dadd_rn(V, vTet);
        M = add3(M, mul3(vTet, cTet));
      }
    }
    if (V <= 0.0) {
      atomicMin(badCell, c);
    } else {
      vol[c] = V;
      st3(cc + 3 * (size_t)c, mul3(1.0 / V, M));
    }
  }
}

// Face centre (point average), area vector by the fan from the first point, unit normal turned
// towards the neighbour (internal) or away from the owner's centroid (boundary).
__global__ void k_face_geom(int nF, int nI, const int* __restrict__ faceOff, const int* __restrict__ facePts,
                            const double* __restrict__ P, const int* __restrict__ owner, const int* __restrict__ neigh,
                            const double* __restrict__ cc, double* xf, double* Af, double* nf, double* Sf,
                            int* badFace) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nF; f += gridDim.x * blockDim.x) {
    const int b0 = faceOff[f], nv = faceOff[f + 1] - b0;
    D3 xfc{0.0, 0.0, 0.0};
    for (int k = 0; k < nv; ++k) xfc = add3(xfc, ld3(P + 3 * (size_t)facePts[b0 + k]));
    xfc = mul3(1.0 / (double)max(nv, 1), xfc);
    st3(xf + 3 * (size_t)f, xfc);
    const D3 a = ld3(P + 3 * (size_t)facePts[b0]);
    D3 area{0.0, 0.0, 0.0};
    for (int i = 1; i + 1 < nv; ++i) {
      const D3 b = ld3(P + 3 * (size_t)facePts[b0 + i]), d = ld3(P + 3 * (size_t)facePts[b0 + i + 1]);
      area = add3(area, mul3(0.5, cross3(sub3(b, a), sub3(d, a))));
    }
    const double mag = __dsqrt_rn(dot3(area, area));
    if (mag <= 1e-30) {
      atomicMin(badFace, f);
      continue;
    }
    D3 n = mul3(1.0 / mag, area);
    const D3 cP = ld3(cc + 3 * (size_t)owner[f]);
    const D3 dt = f < nI ? sub3(ld3(cc + 3 * (size_t)neigh[f]), cP) : sub3(xfc, cP);
    if (dot3(n, dt) < 0.0) n = mul3(-1.0, n);
    Af[f] = mag;
    st3(nf + 3 * (size_t)f, n);
    st3(Sf + 3 * (size_t)f, mul3(mag, n));
  }
}

// Symmetric LSQ moment M = sum w r r^T over the distinct neighbours (ascending) and then the
// boundary faces (ascending) of cell P, w = 1 / max(|r|^2, 1e-30), inverted by cofactors when
// |det| > 1e-20 (else left zero); 6 entries per cell in the input numbering.
__global__ void k_lsq_minv(int nC, const int* __restrict__ off, const int* __restrict__ adj,
                           const int* __restrict__ bOff, const int* __restrict__ bFace, const double* __restrict__ cc,
                           const double* __restrict__ xf, double* minv) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nC; c += gridDim.x * blockDim.x) {
    const D3 xP = ld3(cc + 3 * (size_t)c);
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    auto acc = [&](D3 x) {
      const double r[3] = {__dsub_rn(x.x, xP.x), __dsub_rn(x.y, xP.y), __dsub_rn(x.z, xP.z)};
      const double rr = __dadd_rn(__dadd_rn(__dmul_rn(r[0], r[0]), __dmul_rn(r[1], r[1])), __dmul_rn(r[2], r[2]));
      const double w = 1.0 / fmax(rr, 1e-30);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) M[i][j] = __dadd_rn(M[i][j], __dmul_rn(__dmul_rn(w, r[i]), r[j]));
    };
    for (int k = off[c]; k < off[c + 1]; ++k) acc(ld3(cc + 3 * (size_t)adj[k]));
    for (int k = bOff[c]; k < bOff[c + 1]; ++k) acc(ld3(xf + 3 * (size_t)bFace[k]));
    const double a = M[0][0], b = M[0][1], cq = M[0][2], d = M[1][0], e = M[1][1], f2 = M[1][2], g = M[2][0],
                 h = M[2][1], k = M[2][2];
    const double ekfh = __dsub_rn(__dmul_rn(e, k), __dmul_rn(f2, h));
    const double dkfg = __dsub_rn(__dmul_rn(d, k), __dmul_rn(f2, g));
    const double dheg = __dsub_rn(__dmul_rn(d, h), __dmul_rn(e, g));
    const double det = __dadd_rn(__dsub_rn(__dmul_rn(a, ekfh), __dmul_rn(b, dkfg)), __dmul_rn(cq, dheg));
    double* o = minv + 6 * (size_t)c;
    if (fabs(det) > 1e-20) {
      o[0] = __ddiv_rn(ekfh, det);
      o[1] = __ddiv_rn(__dsub_rn(__dmul_rn(cq, h), __dmul_rn(b, k)), det);
      o[2] = __ddiv_rn(__dsub_rn(__dmul_rn(b, f2), __dmul_rn(cq, e)), det);
      o[3] = __ddiv_rn(__dsub_rn(__dmul_rn(a, k), __dmul_rn(cq, g)), det);
      o[4] = __ddiv_rn(__dsub_rn(__dmul_rn(cq, d), __dmul_rn(a, f2)), det);
      o[5] = __ddiv_rn(__dsub_rn(__dmul_rn(a, e), __dmul_rn(b, d)), det);
    } else {
      for (int q = 0; q < 6; ++q) o[q] = 0.0;
    }
  }
}

// The eight doubles of every slot's face record in slot order (zero and flags 0 on padding).
__global__ void k_slot_geom(size_t nE, const int* __restrict__ slotFace, const FaceRec* __restrict__ face,
                            const uint8_t* __restrict__ fFlags, double* slotGeom, uint8_t* slotFlags) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nE; e += (size_t)gridDim.x * blockDim.x) {
    const int f = slotFace[e];
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint8_t fl = 0;
    if (f >= 0) {
      const FaceRec r = face[f];
      v[0] = r.lam;
      v[1] = r.g;
      v[2] = r.t[0];
      v[3] = r.t[1];
      v[4] = r.t[2];
      v[5] = r.d[0];
      v[6] = r.d[1];
      v[7] = r.d[2];
      fl = fFlags[f];
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) slotGeom[(size_t)q * nE + e] = v[q];
    slotFlags[e] = fl;
  }
}

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e) + " in " + what);
}

// Device buffers freed on scope exit (set-up scratch only).
struct Scratch {
  std::vector<void*> p;
  template <class T>
  T* up(const T* h, size_t n, cudaStream_t s) {
    void* d = nullptr;
    ck(cudaMalloc(&d, std::max<size_t>(n, 1) * sizeof(T)), "set-up allocation");
    p.push_back(d);
    if (n && h) ck(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, s), "set-up upload");
    return static_cast<T*>(d);
  }
  template <class T>
  T* zeros(size_t n, cudaStream_t s) {
    T* d = up<T>(nullptr, n, s);
    ck(cudaMemsetAsync(d, 0, std::max<size_t>(n, 1) * sizeof(T), s), "set-up clear");
    return d;
  }
  ~Scratch() {
    for (void* q : p) cudaFree(q);
  }
};

int grid_for(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

}  // namespace

bool compute_geometry_gpu(HostMesh& m, cudaStream_t s) {
  const int nC = m.nCells, nF = m.nFaces, nI = m.nInternalFaces, nP = m.nPoints();
  for (int f = 0; f < nF; ++f)
    for (int k = m.faceOff[f]; k < m.faceOff[f + 1]; ++k)
      if (m.facePts[k] < 0 || m.facePts[k] >= nP)
        throw std::runtime_error("face " + std::to_string(f) + " references a missing point");
  Scratch sc;
  const double* P = sc.up(m.points.empty() ? nullptr : m.points[0].data(), 3 * (size_t)nP, s);
  const int* faceOff = sc.up(m.faceOff.data(), m.faceOff.size(), s);
  const int* facePts = sc.up(m.facePts.data(), m.facePts.size(), s);
  const int* cfOff = sc.up(m.cellFaceOff.data(), m.cellFaceOff.size(), s);
  const int* cfFace = sc.up(m.cellFaces.data(), m.cellFaces.size(), s);
  const signed char* cfOri = sc.up(m.cellFaceOri.data(), m.cellFaceOri.size(), s);
  const int* own = sc.up(m.owner.data(), m.owner.size(), s);
  const int* nei = sc.up(m.neigh.data(), m.neigh.size(), s);
  double* vol = sc.zeros<double>(nC, s);
  double* cc = sc.zeros<double>(3 * (size_t)nC, s);
  double* xf = sc.zeros<double>(3 * (size_t)nF, s);
  double* Af = sc.zeros<double>(nF, s);
  double* nf = sc.zeros<double>(3 * (size_t)nF, s);
  double* Sf = sc.zeros<double>(3 * (size_t)nF, s);
  int* flags = sc.up<int>(nullptr, 3, s);
  const int init[3] = {INT32_MAX, INT32_MAX, 0};  // bad cell, bad face, overflow
  ck(cudaMemcpyAsync(flags, init, sizeof(init), cudaMemcpyHostToDevice, s), "set-up flags");
  k_cell_geom<<<grid_for(nC), 256, 0, s>>>(nC, cfOff, cfFace, cfOri, faceOff, facePts, P, vol, cc, flags, flags + 2);
  ck(cudaGetLastError(), "cell geometry");
  int h[3];
  ck(cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, s), "set-up flags");
  ck(cudaStreamSynchronize(s), "cell geometry");
  if (h[2]) return false;  // a cell with more distinct points than the kernel holds: host path
  if (h[0] != INT32_MAX) throw std::runtime_error("Non-positive cell volume at cell " + std::to_string(h[0]));
  k_face_geom<<<grid_for(nF), 256, 0, s>>>(nF, nI, faceOff, facePts, P, own, nei, cc, xf, Af, nf, Sf, flags + 1);
  ck(cudaGetLastError(), "face geometry");
  ck(cudaMemcpyAsync(h, flags, sizeof(h), cudaMemcpyDeviceToHost, s), "set-up flags");
  ck(cudaStreamSynchronize(s), "face geometry");
  if (h[1] != INT32_MAX) throw std::runtime_error("Degenerate face area at face " + std::to_string(h[1]));
  m.cc.resize(nC);
  m.vol.resize(nC);
  m.xf.resize(nF);
  m.Af.resize(nF);
  m.nf.resize(nF);
  m.Sf.resize(nF);
  auto down = [&](void* dst, const void* src, size_t bytes) {
    if (bytes) ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "set-up download");
  };
  down(m.cc.data(), cc, 24 * (size_t)nC);
  down(m.vol.data(), vol, 8 * (size_t)nC);
  down(m.xf.data(), xf, 24 * (size_t)nF);
  down(m.Af.data(), Af, 8 * (size_t)nF);
  down(m.nf.data(), nf, 24 * (size_t)nF);
  down(m.Sf.data(), Sf, 24 * (size_t)nF);
  ck(cudaStreamSynchronize(s), "geometry download");
  max_nonorth_deg(m);
  return true;
}

std::vector<double> lsq_minv_gpu(const HostMesh& m, const std::vector<int>& off, const std::vector<int>& adj,
                                 cudaStream_t s) {
  const int nC = m.nCells, nI = m.nInternalFaces, nF = m.nFaces;
  // boundary faces of each cell, ascending (the reference's cellBFace lists)
  std::vector<int> bOff(nC + 1, 0), bFace(nF - nI);
  for (int f = nI; f < nF; ++f) bOff[m.owner[f] + 1]++;
  for (int c = 0; c < nC; ++c) bOff[c + 1] += bOff[c];
  {
    std::vector<int> fill(bOff.begin(), bOff.end() - 1);
    for (int f = nI; f < nF; ++f) bFace[fill[m.owner[f]]++] = f;
  }
  Scratch sc;
  const int* dOff = sc.up(off.data(), off.size(), s);
  const int* dAdj = sc.up(adj.data(), adj.size(), s);
  const int* dbOff = sc.up(bOff.data(), bOff.size(), s);
  const int* dbFace = sc.up(bFace.data(), bFace.size(), s);
  const double* cc = sc.up(m.cc.empty() ? nullptr : m.cc[0].data(), 3 * (size_t)nC, s);
  const double* xf = sc.up(m.xf.empty() ? nullptr : m.xf[0].data(), 3 * (size_t)nF, s);
  double* minv = sc.zeros<double>(6 * (size_t)nC, s);
  k_lsq_minv<<<grid_for(nC), 256, 0, s>>>(nC, dOff, dAdj, dbOff, dbFace, cc, xf, minv);
  ck(cudaGetLastError(), "LSQ moments");
  std::vector<double> out(6 * (size_t)nC);
  if (!out.empty()) ck(cudaMemcpyAsync(out.data(), minv, out.size() * 8, cudaMemcpyDeviceToHost, s), "LSQ download");
  ck(cudaStreamSynchronize(s), "LSQ moments");
  return out;
}

void build_slot_geometry(size_t nE, const int* slotFace, const FaceRec* face, const uint8_t* fFlags, double* slotGeom,
                         uint8_t* slotFlags, cudaStream_t s) {
  k_slot_geom<<<grid_for(nE), 256, 0, s>>>(nE, slotFace, face, fFlags, slotGeom, slotFlags);
  ck(cudaGetLastError(), "slot geometry");
}

}  // namespace anb
