// TEST INFRASTRUCTURE ONLY.  C entry points over the reference's libpoisson, compiled from the
// reference tree by oracle/build_ref.sh (nothing is copied into this repository):
// read_openfoam_polymesh (src/mesh.cu), compute_lsq_gradient (src/gradient.cu) and
// build_scalar_pattern / assemble_scalar_elliptic_system (src/scalar_elliptic.cu).  libscalar's
// entry points are in ref_transport_shim.cu.  The tests compare the oracle's restatement
// (oracle.cpp orc_scalar_*) with these and generate the MMS golden orders
// (tests/golden/make_golden_mms.py).
#include "gradient.h"
#include "mesh.h"
#include "scalar_elliptic.h"

#include <cstring>

namespace {

struct RefScalarMesh {
  Mesh mesh;
  CSRPattern pat;
};

void copy_grad(const std::vector<std::array<double, 3>>& g, double* out, int C) {
  for (int c = 0; c < C; ++c)
    for (int k = 0; k < 3; ++k) out[(size_t)k * C + c] = g[c][k];
}

std::vector<std::array<double, 3>> load_grad(const double* g, int C) {
  std::vector<std::array<double, 3>> out(C);
  for (int c = 0; c < C; ++c) out[c] = {g[c], g[C + c], g[2 * C + c]};
  return out;
}

BoundaryFaceData poisson_bc(const Mesh& m, const int* bt, const double* bv) {
  BoundaryFaceData d;
  d.type.assign(m.nFaces, ScalarBCType::Dirichlet);
  d.value.assign(m.nFaces, 0.0);
  for (int f = m.nInternalFaces; f < m.nFaces; ++f) {
    d.type[f] = bt[f] == 0 ? ScalarBCType::Dirichlet : ScalarBCType::Neumann;
    d.value[f] = bv[f];
  }
  return d;
}

}  // namespace

extern "C" {

void* rsm_open(const char* polyMeshDir, char* err, int errlen) {
  try {
    auto* h = new RefScalarMesh();
    h->mesh = read_openfoam_polymesh(polyMeshDir);
    h->pat = build_scalar_pattern(h->mesh);
    return h;
  } catch (const std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    return nullptr;
  }
}

void rsm_close(void* h) { delete static_cast<RefScalarMesh*>(h); }

void rsm_sizes(void* hv, int* out) {
  auto* h = static_cast<RefScalarMesh*>(hv);
  out[0] = h->mesh.nCells;
  out[1] = h->mesh.nFaces;
  out[2] = h->mesh.nInternalFaces;
  out[3] = h->pat.nnz;
}

void rsm_geometry(void* hv, double* cc, double* vol) {
  auto* h = static_cast<RefScalarMesh*>(hv);
  for (int c = 0; c < h->mesh.nCells; ++c) {
    for (int k = 0; k < 3; ++k) cc[3 * c + k] = h->mesh.cc[c][k];
    vol[c] = h->mesh.vol[c];
  }
}

// CSR pattern of libpoisson (libscalar builds the same one, compared through rst_pattern).
void rsm_pattern(void* hv, int* rowOff, int* cols) {
  auto* h = static_cast<RefScalarMesh*>(hv);
  for (int i = 0; i <= h->pat.nRows; ++i) rowOff[i] = h->pat.rowOffsets[i];
  for (int k = 0; k < h->pat.nnz; ++k) cols[k] = (int)h->pat.cols[k];
}

void rsm_poisson_gradient(void* hv, const int* bt, const double* bv, const double* phi, double* g) {
  auto* h = static_cast<RefScalarMesh*>(hv);
  const Mesh& m = h->mesh;
  std::vector<double> ph(phi, phi + m.nCells);
  std::vector<std::array<double, 3>> grad;
  compute_lsq_gradient(m, ph, poisson_bc(m, bt, bv), grad);
  copy_grad(grad, g, m.nCells);
}

int rsm_poisson_assemble(void* hv, const double* gamma, const double* src, const int* bt, const double* bv,
                         const double* grad, int nonorth, int useRef, int refCell, double refValue,
                         double* values, double* rhs, char* err, int errlen) {
  auto* h = static_cast<RefScalarMesh*>(hv);
  const Mesh& m = h->mesh;
  try {
    std::vector<double> gam(gamma, gamma + m.nFaces), s(src, src + m.nCells);
    std::vector<HYPRE_Complex> v, r;
    assemble_scalar_elliptic_system(m, h->pat, gam, s, poisson_bc(m, bt, bv), load_grad(grad, m.nCells), v, r,
                                    nonorth != 0, useRef != 0, refCell, refValue);
    std::memcpy(values, v.data(), v.size() * sizeof(double));
    std::memcpy(rhs, r.data(), r.size() * sizeof(double));
    return 0;
  } catch (const std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
}

}  // extern "C"
