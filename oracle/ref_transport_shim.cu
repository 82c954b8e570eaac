// TEST INFRASTRUCTURE ONLY.  C entry points over the reference's libscalar, compiled from the
// reference tree by oracle/build_ref.sh (nothing is copied into this repository).  Its helpers
// (build_boundary_face_data, compute_lsq_gradient, build_scalar_pattern,
// assemble_scalar_transport_system) live in an anonymous namespace of
// src/scalar_transport_library.cu, so that translation unit is included here to reach them.
// Meshes come from libpoisson's reader (rsm_open in ref_scalar_shim.cu).
#include "scalar_transport_library.cu"

#include <cstring>

namespace {

void copy_grad(const std::vector<std::array<double, 3>>& g, double* out, int C) {
  for (int c = 0; c < C; ++c)
    for (int k = 0; k < 3; ++k) out[(size_t)k * C + c] = g[c][k];
}

std::vector<std::array<double, 3>> load_grad(const double* g, int C) {
  std::vector<std::array<double, 3>> out(C);
  for (int c = 0; c < C; ++c) out[c] = {g[c], g[C + c], g[2 * C + c]};
  return out;
}

libscalar::BoundaryFaceData transport_bc(const Mesh& m, const int* bt, const double* bv) {
  libscalar::BoundaryFaceData d;
  d.type.assign(m.nFaces, libscalar::ScalarBCType::ZeroGradient);
  d.value.assign(m.nFaces, 0.0);
  for (int f = m.nInternalFaces; f < m.nFaces; ++f) {
    d.type[f] = bt[f] == 0   ? libscalar::ScalarBCType::Dirichlet
                : bt[f] == 2 ? libscalar::ScalarBCType::ZeroGradient
                             : libscalar::ScalarBCType::NeumannGradient;
    d.value[f] = bv[f];
  }
  return d;
}

// The mesh handle of ref_scalar_shim.cu starts with the Mesh.
const Mesh& mesh_of(void* h) { return *static_cast<const Mesh*>(h); }

}  // namespace

extern "C" {

void rst_pattern(void* hv, int* rowOff, int* cols) {
  const auto pat = libscalar::build_scalar_pattern(mesh_of(hv));
  for (int i = 0; i <= pat.nRows; ++i) rowOff[i] = pat.rowOffsets[i];
  for (int k = 0; k < pat.nnz; ++k) cols[k] = (int)pat.cols[k];
}

void rst_gradient(void* hv, const int* bt, const double* bv, const double* phi, double* g) {
  const Mesh& m = mesh_of(hv);
  std::vector<double> ph(phi, phi + m.nCells);
  std::vector<std::array<double, 3>> grad;
  libscalar::compute_lsq_gradient(m, ph, transport_bc(m, bt, bv), grad);
  copy_grad(grad, g, m.nCells);
}

int rst_assemble(void* hv, const double* flux, const double* gamma, const double* su, const double* sp,
                           const int* bt, const double* bv, const double* grad, int upwind, int nonorth,
                           double* values, double* rhs, char* err, int errlen) {
  const Mesh& m = mesh_of(hv);
  try {
    libscalar::ScalarTransportInputs in;
    in.faceFlux.assign(flux, flux + m.nFaces);
    in.gammaFace.assign(gamma, gamma + m.nFaces);
    in.Su.assign(su, su + m.nCells);
    in.Sp.assign(sp, sp + m.nCells);
    libscalar::ScalarTransportOptions opt;
    opt.convectionScheme = upwind ? libscalar::ConvectionScheme::Upwind : libscalar::ConvectionScheme::Central;
    opt.diffusionScheme = nonorth ? libscalar::DiffusionScheme::NonOrth : libscalar::DiffusionScheme::Orth;
    std::vector<HYPRE_Complex> v, r;
    libscalar::assemble_scalar_transport_system(m, libscalar::build_scalar_pattern(m), in, transport_bc(m, bt, bv), load_grad(grad, m.nCells),
                                                opt, v, r);
    std::memcpy(values, v.data(), v.size() * sizeof(double));
    std::memcpy(rhs, r.data(), r.size() * sizeof(double));
    return 0;
  } catch (const std::exception& e) {
    std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
}

}  // extern "C"
