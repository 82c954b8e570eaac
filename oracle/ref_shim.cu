// TEST INFRASTRUCTURE ONLY.  C entry points into the reference's own host code.
//
// The reference's apps/generic_simple_v1/src/main.cu is compiled here as-is, from where it lies in
// the reference tree (oracle/build_ref.sh passes its directory as an include path), with the
// single-rank MPI and HYPRE stand-ins of oracle/ref_stubs.  Its file-static host functions are
// reachable from this translation unit, so the tests can run the reference's geometry, LSQ
// gradient, Rhie-Chow flux, continuity, non-orthogonal flux, flux correction, force integral,
// VTU writer and .case expansion on the same inputs as the oracle and the B200 library.
#define main gsv1_reference_main
#include "main.cu"
#undef main

#include <cstring>

namespace {
struct RefMesh {
  Mesh m;
};
std::vector<std::string> types_of(const int* t, int n) {
  std::vector<std::string> s(n);
  for (int i = 0; i < n; ++i) s[i] = t[i] == 1 ? "Dirichlet" : "Neumann";
  return s;
}
std::vector<std::array<double, 3>> aos3(const double* g, int n) {
  std::vector<std::array<double, 3>> v(n);
  for (int i = 0; i < n; ++i) v[i] = {g[3 * i], g[3 * i + 1], g[3 * i + 2]};
  return v;
}
int seterr(char* b, int n, const char* m) {
  if (b && n > 0) std::snprintf(b, n, "%s", m);
  return 1;
}
}  // namespace

extern "C" {

void* ref_read_mesh(const char* dir, char* err, int errlen) {
  try {
    auto* r = new RefMesh();
    r->m = read_openfoam_polymesh(dir);
    return r;
  } catch (const std::exception& e) {
    seterr(err, errlen, e.what());
    return nullptr;
  }
}
void ref_free_mesh(void* h) { delete static_cast<RefMesh*>(h); }
void ref_mesh_sizes(void* h, int* s) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  s[0] = (int)m.P.size();
  s[1] = m.nFaces;
  s[2] = m.nInternalFaces;
  s[3] = m.nCells;
  s[4] = (int)m.patchNames.size();
}
void ref_mesh_geometry(void* h, double* cc, double* vol, double* xf, double* nf, double* sf, double* af, double* mx) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  for (int c = 0; c < m.nCells; ++c) {
    for (int k = 0; k < 3; ++k) cc[3 * c + k] = m.cc[c][k];
    vol[c] = m.vol[c];
  }
  for (int f = 0; f < m.nFaces; ++f) {
    for (int k = 0; k < 3; ++k) {
      xf[3 * f + k] = m.xf[f][k];
      nf[3 * f + k] = m.nf[f][k];
      sf[3 * f + k] = m.Sf[f][k];
    }
    af[f] = m.Af[f];
  }
  *mx = m.maxNonOrthDeg;
}
// compute_lsq_gradient (main.cu:601-618); grad: 3 per cell
void ref_lsq_gradient(void* h, const int* patchType, const double* faceVal, const double* phi, double* grad) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  std::vector<double> ph(phi, phi + m.nCells), fv(faceVal, faceVal + m.nFaces);
  std::vector<std::array<double, 3>> g;
  compute_lsq_gradient(m, ph, types_of(patchType, (int)m.patchNames.size()), fv, g);
  for (int c = 0; c < m.nCells; ++c)
    for (int k = 0; k < 3; ++k) grad[3 * c + k] = g[c][k];
}
// build_rhiechow_predicted_flux_stokes_3d (main.cu:644-716)
void ref_rhie_chow(void* h, const double* u, const double* v, const double* w, const double* p, const double* gradP,
                   const double* rau, const int* tu, const double* uf, const int* tv, const double* vf, const int* tw,
                   const double* wf, double rho, double* phiStar) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  const int C = m.nCells, F = m.nFaces, P = (int)m.patchNames.size();
  std::vector<double> ps;
  build_rhiechow_predicted_flux_stokes_3d(
      m, std::vector<double>(u, u + C), std::vector<double>(v, v + C), std::vector<double>(w, w + C),
      std::vector<double>(p, p + C), aos3(gradP, C), std::vector<double>(rau, rau + C), types_of(tu, P),
      std::vector<double>(uf, uf + F), types_of(tv, P), std::vector<double>(vf, vf + F), types_of(tw, P),
      std::vector<double>(wf, wf + F), rho, ps);
  std::memcpy(phiStar, ps.data(), sizeof(double) * F);
}
// continuity_residual (main.cu:718-728)
void ref_continuity(void* h, const double* phi, double* div) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  std::vector<double> d;
  continuity_residual(m, std::vector<double>(phi, phi + m.nFaces), d);
  std::memcpy(div, d.data(), sizeof(double) * m.nCells);
}
// pressure_nonorth_flux_and_divergence (main.cu:744-789)
void ref_nonorth(void* h, const double* rau, const int* tp, const double* gradP, double* phiNO, double* divNO) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  std::vector<double> a, b;
  pressure_nonorth_flux_and_divergence(m, std::vector<double>(rau, rau + m.nCells),
                                       types_of(tp, (int)m.patchNames.size()), aos3(gradP, m.nCells), a, b);
  std::memcpy(phiNO, a.data(), sizeof(double) * m.nFaces);
  std::memcpy(divNO, b.data(), sizeof(double) * m.nCells);
}
// correct_face_fluxes_simple_nonorth (main.cu:791-829)
void ref_flux_correct(void* h, const double* rau, const int* tp, const double* pFace, const double* phiStar,
                      const double* pCorr, const double* gradP, double* phi) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  const int C = m.nCells, F = m.nFaces;
  std::vector<double> out;
  correct_face_fluxes_simple_nonorth(m, std::vector<double>(rau, rau + C), types_of(tp, (int)m.patchNames.size()),
                                     std::vector<double>(pFace, pFace + F), std::vector<double>(phiStar, phiStar + F),
                                     std::vector<double>(pCorr, pCorr + C), aos3(gradP, C), out);
  std::memcpy(phi, out.data(), sizeof(double) * F);
}
// compute_patch_forces_wall_shear (main.cu:2828-2933); out: Fp[3] Fv[3] F[3] area nFaces
void ref_patch_force(void* h, int patch, const double* u, const double* v, const double* w, const double* p, double rho,
                     double mu, int sign, double* out) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  const int C = m.nCells;
  PatchForceReport r = compute_patch_forces_wall_shear(
      m, patch, std::vector<double>(u, u + C), std::vector<double>(v, v + C), std::vector<double>(w, w + C),
      std::vector<double>(p, p + C), rho, mu, sign, -1.0, -1.0, {{1, 0, 0}}, {{0, 1, 0}}, {{0, 0, 1}});
  for (int d = 0; d < 3; ++d) {
    out[d] = r.Fp[d];
    out[3 + d] = r.Fv[d];
    out[6 + d] = r.F[d];
  }
  out[9] = r.area;
  out[10] = r.nFaces;
}
// write_vtu_polyhedron_cell_data (main.cu:975-983) with the fields of main.cu:3838-3842
int ref_write_vtu(void* h, const char* fn, const double* u, const double* v, const double* w, const double* p) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  const int C = m.nCells;
  std::vector<std::array<double, 3>> U(C);
  std::vector<double> umag(C), pp(p, p + C), divCorr(C, 0.0);
  for (int c = 0; c < C; ++c) {
    U[c] = {u[c], v[c], w[c]};
    umag[c] = std::sqrt(u[c] * u[c] + v[c] * v[c] + w[c] * w[c]);
  }
  try {
    write_vtu_polyhedron_cell_data(fn, m, {"p", "umag", "cell_volume", "divCorr"}, {pp, umag, m.vol, divCorr}, "U", &U);
  } catch (...) {
    return 1;
  }
  return 0;
}
// expand_case_config_args (main.cu:162-331): NUL-separated output, returns the count or -1
int ref_expand_case(int argc, char** argv, char* out, int outlen, char* err, int errlen) {
  try {
    auto r = expand_case_config_args(argc, argv);
    size_t o = 0;
    for (const auto& s : r) {
      if ((int)(o + s.size() + 1) > outlen) return -1;
      std::memcpy(out + o, s.c_str(), s.size() + 1);
      o += s.size() + 1;
    }
    return (int)r.size();
  } catch (const std::exception& e) {
    seterr(err, errlen, e.what());
    return -1;
  }
}
// load_runtime_bc_config + validate + build_patch_geometry_table + apply_bc_specs_to_legacy_face_arrays
int ref_bc_eval(void* h, const char* path, int* tu, int* tv, int* tw, int* tp, double* u, double* v, double* w,
                double* p, char* err, int errlen) {
  const Mesh& m = static_cast<RefMesh*>(h)->m;
  try {
    pipebc::PatchGeometryInput gi;
    gi.nInternalFaces = m.nInternalFaces;
    gi.nFaces = m.nFaces;
    gi.xf = &m.xf;
    gi.nf = &m.nf;
    gi.Sf = &m.Sf;
    gi.Af = &m.Af;
    gi.patchNames = &m.patchNames;
    gi.patchStartFace = &m.patchStartFace;
    gi.patchNFaces = &m.patchNFaces;
    auto table = pipebc::build_patch_geometry_table(gi);
    auto cfg = pipebc::load_runtime_bc_config(path);
    pipebc::validate_runtime_bc_config_against_patches(cfg, m.patchNames);
    pipebc::LegacyBCMeshView lv;
    lv.nFaces = m.nFaces;
    lv.nInternalFaces = m.nInternalFaces;
    lv.patchNames = &m.patchNames;
    lv.patchStartFace = &m.patchStartFace;
    lv.patchNFaces = &m.patchNFaces;
    lv.xf = &m.xf;
    lv.nf = &m.nf;
    const int P = (int)m.patchNames.size();
    std::vector<std::string> a(P, "Neumann"), b(P, "Neumann"), c(P, "Neumann"), d(P, "Neumann");
    std::vector<double> fu(m.nFaces, 0.0), fv(m.nFaces, 0.0), fw(m.nFaces, 0.0), fp(m.nFaces, 0.0);
    pipebc::apply_bc_specs_to_legacy_face_arrays(lv, table, cfg.velocityPatchSpecs, cfg.pressurePatchSpecs, 0.0, a, b,
                                                 c, d, fu, fv, fw, fp);
    for (int k = 0; k < P; ++k) {
      tu[k] = bc_to_int(a[k]);
      tv[k] = bc_to_int(b[k]);
      tw[k] = bc_to_int(c[k]);
      tp[k] = bc_to_int(d[k]);
    }
    std::memcpy(u, fu.data(), sizeof(double) * m.nFaces);
    std::memcpy(v, fv.data(), sizeof(double) * m.nFaces);
    std::memcpy(w, fw.data(), sizeof(double) * m.nFaces);
    std::memcpy(p, fp.data(), sizeof(double) * m.nFaces);
    return 0;
  } catch (const std::exception& e) {
    return seterr(err, errlen, e.what());
  }
}

}  // extern "C"
