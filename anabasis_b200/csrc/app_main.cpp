// anabasis_simple: drop-in replacement of the reference's generic_simple_v1 executable.
//
// Same command line (-case-config <file> [flags]), .case keys, .bc grammar, polyMesh reader,
// stdout lines, <outPrefix>_final.vtu / _iterNNNNNN.vtu and <outPrefix>_summary.txt as
// apps/generic_simple_v1/src/main.cu:2936-3915; the SIMPLE iterations run in libanb.so on one
// GPU.  Errors print the reference's message and exit with status 1 (the reference aborts
// through MPI_Abort or an uncaught exception).
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/anb.h"
#include "host_case.hpp"
#include "host_mesh.hpp"
#include "host_output.hpp"

using namespace anb;

namespace {

[[noreturn]] void die(const std::string& msg, int code = 1) {
  std::fprintf(stderr, "%s\n", msg.c_str());
  std::exit(code);
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

std::array<double, 3> normalized(std::array<double, 3> v) {
  const double m = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (m <= 1.0e-300) return {0, 0, 0};
  return {v[0] / m, v[1] / m, v[2] / m};
}

void print_patch(const PatchGeom& g) {
  std::printf("Patch summary [%s]\n", g.name.c_str());
  std::printf("  faces      : %d\n", g.nFaces);
  std::printf("  area       : %.12e\n", g.totalArea);
  std::printf("  centroid   : [%.6e, %.6e, %.6e]\n", g.centroid[0], g.centroid[1], g.centroid[2]);
  std::printf("  avg normal : [%.6e, %.6e, %.6e]\n", g.averageNormal[0], g.averageNormal[1], g.averageNormal[2]);
  std::printf("  planarity  : %.6f\n", g.planarity);
}

// compute_cylinder_forces_paper / _vector_wall_shear, main.cu:883-973 and 2707-2785 (host).
struct CylForce {
  bool valid = false;
  std::string name;
  int nFaces = 0;
  double area = 0, FDp = 0, FDv = 0, FLp = 0, FLv = 0, CD = 0, CL = 0, denom = 0;
  double minDn = 1e300, maxDn = 0, maxDvt = 0;
  std::array<double, 3> Fp{{0, 0, 0}}, Fv{{0, 0, 0}}, F{{0, 0, 0}}, Cv{{0, 0, 0}};
  double vminDn = 1e300, vmaxDn = 0, maxUt = 0, maxShear = 0;
};

CylForce cylinder_forces(const HostMesh& m, int patch, const std::vector<double>& u, const std::vector<double>& v,
                         const std::vector<double>& w, const std::vector<double>& p, double rho, double mu, double D,
                         double H, double Ubar) {
  CylForce r;
  r.valid = true;
  r.name = m.patches[patch].name;
  r.denom = rho * Ubar * Ubar * D * H;
  const int f0 = m.patches[patch].start, f1 = f0 + m.patches[patch].nFaces;
  for (int f = f0; f < f1; ++f) {  // paper formula
    const int P = m.owner[f];
    const double A = m.Af[f];
    if (A <= 1e-300) continue;
    std::array<double, 3> n{{-m.nf[f][0], -m.nf[f][1], -m.nf[f][2]}};
    double nm = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (nm <= 1e-300) continue;
    for (auto& x : n) x *= 1.0 / nm;
    std::array<double, 3> t{{n[1], -n[0], 0.0}};
    double tm = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    if (tm <= 1e-14) continue;
    for (auto& x : t) x *= 1.0 / tm;
    const double vt = u[P] * t[0] + v[P] * t[1] + w[P] * t[2];
    std::array<double, 3> dx{{m.cc[P][0] - m.xf[f][0], m.cc[P][1] - m.xf[f][1], m.cc[P][2] - m.xf[f][2]}};
    double dn = dx[0] * n[0] + dx[1] * n[1] + dx[2] * n[2];
    if (dn <= 1e-14) dn = std::fabs(dn);
    if (dn <= 1e-14) dn = std::sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    if (dn <= 1e-14) continue;
    const double dvt = vt / dn;
    r.FDp += (-p[P] * n[0]) * A;
    r.FDv += (mu * dvt * n[1]) * A;
    r.FLp += (-p[P] * n[1]) * A;
    r.FLv += (-mu * dvt * n[0]) * A;
    r.area += A;
    r.nFaces += 1;
    r.minDn = std::min(r.minDn, dn);
    r.maxDn = std::max(r.maxDn, dn);
    r.maxDvt = std::max(r.maxDvt, std::fabs(dvt));
  }
  if (r.denom > 1e-300) {
    r.CD = 2.0 * (r.FDp + r.FDv) / r.denom;
    r.CL = 2.0 * (r.FLp + r.FLv) / r.denom;
  }
  if (r.minDn == 1e300) r.minDn = 0.0;
  for (int f = f0; f < f1; ++f) {  // vector wall-shear traction
    const int P = m.owner[f];
    const double A = m.Af[f];
    if (A <= 1e-300) continue;
    std::array<double, 3> n{{-m.nf[f][0], -m.nf[f][1], -m.nf[f][2]}};
    double nm = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (nm <= 1e-300) continue;
    for (auto& x : n) x *= 1.0 / nm;
    std::array<double, 3> dx{{m.cc[P][0] - m.xf[f][0], m.cc[P][1] - m.xf[f][1], m.cc[P][2] - m.xf[f][2]}};
    double dn = dx[0] * n[0] + dx[1] * n[1] + dx[2] * n[2];
    if (dn <= 1e-14) dn = std::fabs(dn);
    if (dn <= 1e-14) dn = std::sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    if (dn <= 1e-14) continue;
    std::array<double, 3> U{{u[P], v[P], w[P]}};
    const double Un = U[0] * n[0] + U[1] * n[1] + U[2] * n[2];
    std::array<double, 3> Ut{{U[0] - Un * n[0], U[1] - Un * n[1], U[2] - Un * n[2]}};
    const double Utm = std::sqrt(Ut[0] * Ut[0] + Ut[1] * Ut[1] + Ut[2] * Ut[2]);
    for (int d = 0; d < 3; ++d) {
      const double fp = -p[P] * n[d] * A, fv = mu * Ut[d] / dn * A;
      r.Fp[d] += fp;
      r.Fv[d] += fv;
      r.F[d] += fp + fv;
    }
    r.vminDn = std::min(r.vminDn, dn);
    r.vmaxDn = std::max(r.vmaxDn, dn);
    r.maxUt = std::max(r.maxUt, Utm);
    r.maxShear = std::max(r.maxShear, mu * Utm / dn);
  }
  if (r.denom > 1e-300)
    for (int d = 0; d < 3; ++d) r.Cv[d] = 2.0 * r.F[d] / r.denom;
  if (r.vminDn == 1e300) r.vminDn = 0.0;
  return r;
}

void write_vtu_fields(const HostMesh& m, const std::string& fn, const std::vector<double>& u,
                      const std::vector<double>& v, const std::vector<double>& w, const std::vector<double>& p,
                      const std::vector<double>& divCorr, bool binary) {
  std::vector<double> umag(m.nCells);
  for (int c = 0; c < m.nCells; ++c) umag[c] = std::sqrt(u[c] * u[c] + v[c] * v[c] + w[c] * w[c]);
  const double* vec[3] = {u.data(), v.data(), w.data()};
  const std::vector<std::string> names = {"p", "umag", "cell_volume", "divCorr"};
  const std::vector<const double*> data = {p.data(), umag.data(), m.vol.data(), divCorr.data()};
  if (binary) write_vtu_appended(m, fn, names, data, "U", vec);
  else write_vtu(m, fn, names, data, "U", vec);
}

}  // namespace

int main(int argc, char** argv) {
  Params par;
  try {
    std::vector<std::string> a(argv, argv + argc);
    parse_args(expand_case_config_args(a), par);
  } catch (const CliError& e) {
    die(e.what(), e.code);
  } catch (const std::exception& e) {
    die(e.what());
  }
  if (cudaSetDevice(par.device) != cudaSuccess) die("CUDA ERROR: cannot select device " + std::to_string(par.device));
  {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, par.device) != cudaSuccess) die("CUDA ERROR: no device properties");
    std::printf("Running on \"%s\", major %d, minor %d, total memory %.2f GiB\n", prop.name, prop.major, prop.minor,
                (double)prop.totalGlobalMem / (1024.0 * 1024.0 * 1024.0));
  }
  HostMesh mesh;
  try {
    mesh = read_polymesh(par.polyMeshDir);
  } catch (const std::exception& e) {
    die(e.what());
  }
  double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300, zmin = 1e300, zmax = -1e300, vmin = 1e300, vmax = -1e300;
  for (const auto& p : mesh.points) {
    xmin = std::min(xmin, p[0]); xmax = std::max(xmax, p[0]);
    ymin = std::min(ymin, p[1]); ymax = std::max(ymax, p[1]);
    zmin = std::min(zmin, p[2]); zmax = std::max(zmax, p[2]);
  }
  for (double v : mesh.vol) { vmin = std::min(vmin, v); vmax = std::max(vmax, v); }
  int wallPatch = -1, inletPatch = -1, outletPatch = -1, cylinderPatch = -1;
  for (size_t k = 0; k < mesh.patches.size(); ++k) {
    if (mesh.patches[k].name == par.wallPatchName) wallPatch = (int)k;
    if (mesh.patches[k].name == "patch_3_0") cylinderPatch = (int)k;
    if (mesh.patches[k].name == par.inletPatchName) inletPatch = (int)k;
    if (mesh.patches[k].name == par.outletPatchName) outletPatch = (int)k;
  }
  if (wallPatch < 0 || inletPatch < 0 || outletPatch < 0) die("Could not find wall/inlet/outlet patch.");
  const double mu = par.muExplicit ? par.mu : (par.rho * par.Umean * par.pipeDiameter / par.Re);
  std::printf("============================================================\n");
  std::printf("generic_simple_v1: OpenFOAM polyMesh SIMPLE solver\n");
  std::printf("anabasis_b200: B200 SIMPLE library (atomic-free face loops, aggregation-AMG PCG, BiCGSTAB)\n");
  std::printf("============================================================\n");
  std::printf("polyMeshDir : %s\n", par.polyMeshDir.c_str());
  std::printf("outPrefix   : %s\n", par.outPrefix.c_str());
  std::printf("------------------------------------------------------------\n");
  std::printf("Points         : %d\n", mesh.nPoints());
  std::printf("Faces          : %d\n", mesh.nFaces);
  std::printf("Internal faces : %d\n", mesh.nInternalFaces);
  std::printf("Cells          : %d\n", mesh.nCells);
  std::printf("BBox           : [%g, %g] x [%g, %g] x [%g, %g]\n", xmin, xmax, ymin, ymax, zmin, zmax);
  std::printf("Volume min/max : %.8e / %.8e\n", vmin, vmax);
  std::printf("maxNonOrthDeg  : %.6f\n", mesh.maxNonOrthDeg);
  std::printf("Momentum solve : SELL-32 BiCGSTAB + Jacobi (device)\n");
  std::printf("Pressure solve : SELL-32 PCG + %s (device)\n", par.p_use_amg ? "aggregation AMG" : "Jacobi");
  std::printf("rho            : %.8g\n", par.rho);
  std::printf("Re             : %.8g\n", par.Re);
  std::printf("Umean          : %.8g\n", par.Umean);
  std::printf("pipeDiameter   : %.8g\n", par.pipeDiameter);
  std::printf("pipeLength     : %.8g\n", par.pipeLength);
  std::printf("wall/in/out    : %s / %s / %s\n", par.wallPatchName.c_str(), par.inletPatchName.c_str(), par.outletPatchName.c_str());
  std::printf("mu             : %.8e\n", mu);
  std::printf("mu source      : %s\n", par.muExplicit ? "direct -mu / case mu" : "legacy rho*Umean*pipeD/Re");
  std::printf("steady mode    : ON (no pseudo-time mass term)\n");
  std::printf("nsteps         : %d\n", par.nsteps);
  std::printf("nVelNonOrthCorr: %d\n", par.nVelNonOrthCorr);
  std::printf("nNonOrthCorr   : %d\n", par.nNonOrthCorr);
  std::printf("nPressureCorr  : %d\n", par.nPressureCorr);
  std::printf("velTol / velRelTol : %.3e / %.3e\n", par.velTol, par.velRelTol);
  std::printf("pTol   / pRelTol   : %.3e / %.3e\n", par.pTol, par.pRelTol);
  std::printf("pAmgRebuildEvery   : %d\n", par.pAmgRebuildEvery);
  std::printf("precision          : %s\n", par.precision ? "mixed" : "fp64");
  std::printf("------------------------------------------------------------\n");
  if (par.bcConfigPath.empty())
    die("generic_simple_v1 requires explicit runtime BCs.\nAdd velocity/pressure lines to the case file, or set bcConfig.");
  BCConfig cfg;
  std::vector<PatchGeom> geom;
  FaceBC bc;
  try {
    geom = build_patch_geometry(mesh);
    cfg = load_bc_config(par.bcConfigPath);
    std::vector<std::string> names;
    for (const auto& p : mesh.patches) names.push_back(p.name);
    validate_bc_config(cfg, names);
  } catch (const std::exception& e) {
    die(e.what());
  }
  auto dv = duplicate_velocity_patches(cfg);
  if (!dv.empty()) {
    std::fprintf(stderr, "Duplicate velocity BC specs found:\n");
    for (auto& n : dv) std::fprintf(stderr, "  %s\n", n.c_str());
    std::exit(1);
  }
  auto dp = duplicate_pressure_patches(cfg);
  if (!dp.empty()) {
    std::fprintf(stderr, "Duplicate pressure BC specs found:\n");
    for (auto& n : dp) std::fprintf(stderr, "  %s\n", n.c_str());
    std::exit(1);
  }
  std::printf("------------------------------------------------------------\n");
  std::printf("All mesh patches detected in polyMesh:\n");
  for (const auto& g : geom) print_patch(g);
  std::printf("------------------------------------------------------------\n");
  std::printf("Runtime BC patch coverage:\n");
  std::vector<std::string> missV, missP;
  for (const auto& pi : mesh.patches) {
    bool hv = false, hp = false;
    for (const auto& s : cfg.vel) hv = hv || s.patch == pi.name;
    for (const auto& s : cfg.pres) hp = hp || s.patch == pi.name;
    std::printf("  %-32s velocity=%s pressure=%s\n", pi.name.c_str(), hv ? "yes" : "NO", hp ? "yes" : "NO");
    if (!hv) missV.push_back(pi.name);
    if (!hp) missP.push_back(pi.name);
  }
  if (!missV.empty() || !missP.empty()) {
    std::fprintf(stderr, "\nERROR: incomplete runtime BC coverage.\n");
    if (!missV.empty()) {
      std::fprintf(stderr, "Missing velocity BC for patches:\n");
      for (auto& n : missV) std::fprintf(stderr, "  %s\n", n.c_str());
    }
    if (!missP.empty()) {
      std::fprintf(stderr, "Missing pressure BC for patches:\n");
      for (auto& n : missP) std::fprintf(stderr, "  %s\n", n.c_str());
    }
    std::fprintf(stderr,
                 "\nEvery polyMesh boundary patch must have exactly one velocity BC and one pressure BC in generic_simple_v1.\n");
    std::exit(1);
  }
  const bool pRefNeeded = pressure_reference_required(cfg);
  print_patch(geom[wallPatch]);
  if (cylinderPatch >= 0) print_patch(geom[cylinderPatch]);
  print_patch(geom[inletPatch]);
  print_patch(geom[outletPatch]);
  std::printf("Pressure reference required: %s\n", pRefNeeded ? "yes" : "no");
  std::printf("BC config source         : %s\n", par.bcConfigPath.c_str());
  int inletCount = 0;
  for (int f = mesh.nInternalFaces; f < mesh.nFaces; ++f)
    if (mesh.bPatch[f] - 1 == inletPatch) ++inletCount;
  if (inletCount <= 0) die("Inlet patch has no boundary faces.");
  try {
    bc = evaluate_face_bc(mesh, geom, cfg);
  } catch (const std::exception& e) {
    die(e.what());
  }
  // initial velocity: mean of the inlet face values (main.cu:3302-3322), p = 0
  double iu = 0, iv = 0, iw = 0;
  int ic = 0;
  for (int f = mesh.nInternalFaces; f < mesh.nFaces; ++f)
    if (mesh.bPatch[f] - 1 == inletPatch) {
      iu += bc.u[f]; iv += bc.v[f]; iw += bc.w[f];
      ++ic;
    }
  if (ic > 0) { iu /= ic; iv /= ic; iw /= ic; }
  std::vector<double> u(mesh.nCells, iu), v(mesh.nCells, iv), w(mesh.nCells, iw), p(mesh.nCells, 0.0);
  std::vector<double> divCorr(mesh.nCells, 0.0);  // written as zeros, like the reference (main.cu:3327)

  anb_params prm;
  anb_default_params(&prm);
  prm.rho = par.rho;
  prm.mu = mu;
  prm.u_relax = par.uRelax;
  prm.p_relax = par.pRelax;
  prm.n_nonorth_corr = par.nNonOrthCorr;
  prm.n_vel_nonorth_corr = par.nVelNonOrthCorr;
  prm.n_pressure_corr = par.nPressureCorr;
  prm.vel_maxit = par.velMaxit;
  prm.vel_tol = par.velTol;
  prm.vel_rel_tol = par.velRelTol;
  prm.p_maxit = par.pMaxit;
  prm.p_tol = par.pTol;
  prm.p_rel_tol = par.pRelTol;
  prm.corr_tol = par.corrTol;
  prm.p_amg_rebuild_every = par.pAmgRebuildEvery;
  prm.p_use_amg = par.p_use_amg;
  prm.p_amg_setup_scope = par.pAmgSetupScope;
  prm.precision = par.precision;
  prm.device = par.device;
  std::vector<double> pts((size_t)3 * mesh.nPoints());
  for (int i = 0; i < mesh.nPoints(); ++i)
    for (int k = 0; k < 3; ++k) pts[3 * i + k] = mesh.points[i][k];
  std::vector<int> ps(mesh.patches.size()), pn(mesh.patches.size());
  for (size_t k = 0; k < mesh.patches.size(); ++k) {
    ps[k] = mesh.patches[k].start;
    pn[k] = mesh.patches[k].nFaces;
  }
  anb_mesh_desc md{mesh.nPoints(), pts.data(), mesh.nFaces, mesh.faceOff.data(), mesh.facePts.data(),
                   mesh.nInternalFaces, mesh.owner.data(), mesh.neigh.data(), (int)mesh.patches.size(),
                   ps.data(), pn.data()};
  anb_ctx* ctx = nullptr;
  const double tSetup0 = now();
  if (anb_create(&md, &prm, &ctx) != ANB_OK) die(std::string("anb_create: ") + anb_last_error(nullptr));
  if (anb_set_bc(ctx, bc.typeU.data(), bc.typeV.data(), bc.typeW.data(), bc.typeP.data(), bc.u.data(), bc.v.data(),
                 bc.w.data(), bc.p.data()) != ANB_OK ||
      anb_set_state(ctx, u.data(), v.data(), w.data(), p.data()) != ANB_OK)
    die(std::string("anb setup: ") + anb_last_error(ctx));
  const double tSetup = now() - tSetup0;

  int stepConverged = 0;
  anb_iter_stats last{};
  double runStart = now();
  double gpuSeconds = 0.0;
  int pcgTotal = 0;
  for (int step = 1; step <= par.nsteps; ++step) {
    const double it0 = now();
    anb_iter_stats st{};
    int done = 0;
    int rc = anb_simple_iterate(ctx, 1, -1.0, -1.0, &st, &done);
    if (rc == ANB_NOT_CONVERGED)
      std::fprintf(stderr, "WARNING: inner solve non-convergence at iteration %d. Continuing.\n", step);
    else if (rc != ANB_OK && rc != ANB_ERR_DIVERGED)
      die(std::string("anb_simple_iterate: ") + anb_last_error(ctx));
    last = st;
    gpuSeconds += st.iter_seconds;
    pcgTotal = st.its_p_total;
    const double iterWall = now() - it0, totalWall = now() - runStart;
    if (step == 1 || (par.printEvery > 0 && step % par.printEvery == 0))
      std::printf(
          "iter %4d : massRes = %.3e, duRel = %.3e, dvRel = %.3e, dwRel = %.3e, dpRel = %.3e, bicgstab=[%d %d %d], "
          "pcgLast=%d, pcgTot=%d, iterWall = %.3e s, totalWall = %.3e s\n",
          step, st.mass_res, st.du_rel, st.dv_rel, st.dw_rel, st.dp_rel, st.its_u, st.its_v, st.its_w,
          st.its_p_last, pcgTotal, iterWall, totalWall);
    if (par.writeEvery > 0 && step % par.writeEvery == 0 && par.write_vtu) {
      anb_get_state(ctx, u.data(), v.data(), w.data(), p.data(), nullptr);
      std::ostringstream oss;
      oss << par.outPrefix << "_iter" << std::setw(6) << std::setfill('0') << step << ".vtu";
      write_vtu_fields(mesh, oss.str(), u, v, w, p, divCorr, par.vtuBinary != 0);
    }
    if (!std::isfinite(st.mass_res) || st.mass_res > 1e50) {
      std::fprintf(stderr, "SIMPLE-like steady solve diverged.\n");
      break;
    }
    if (st.mass_res < par.tolMass && std::max({st.du_rel, st.dv_rel, st.dw_rel}) < par.tolVel) {
      stepConverged = step;
      std::printf("Converged at iteration %d : massRes = %.3e\n", step, st.mass_res);
      break;
    }
    stepConverged = step;
  }
  const double loopWall = now() - runStart;
  anb_get_state(ctx, u.data(), v.data(), w.data(), p.data(), nullptr);
  double umax = 0, vmaxf = 0, wmaxf = 0, pmax = 0;
  for (int c = 0; c < mesh.nCells; ++c) {
    umax = std::max(umax, std::fabs(u[c]));
    vmaxf = std::max(vmaxf, std::fabs(v[c]));
    wmaxf = std::max(wmaxf, std::fabs(w[c]));
    pmax = std::max(pmax, std::fabs(p[c]));
  }
  CylForce cyl;
  if (cylinderPatch >= 0)
    cyl = cylinder_forces(mesh, cylinderPatch, u, v, w, p, par.rho, mu, par.pipeDiameter, 0.41, (4.0 / 9.0) * par.Umean);
  anb_force_report pf{};
  int forcePatch = -1;
  if (par.forceEnable) {
    for (size_t k = 0; k < mesh.patches.size(); ++k)
      if (mesh.patches[k].name == par.forcePatchName) forcePatch = (int)k;
    anb_patch_force(ctx, forcePatch, par.forceNormalSign, &pf);
  }
  const auto dragDir = normalized(par.forceDragDir);
  (void)dragDir;
  std::printf("\nFinal summary:\n");
  std::printf("------------------------------------------------------------\n");
  std::printf("Iterations    = %d\n", stepConverged);
  std::printf("massRes       = %.8e\n", last.mass_res);
  std::printf("max|u|        = %.8e\n", umax);
  std::printf("max|v|        = %.8e\n", vmaxf);
  std::printf("max|w|        = %.8e\n", wmaxf);
  std::printf("max|p|        = %.8e\n", pmax);
  if (cyl.valid) {
    std::printf("------------------------------------------------------------\n");
    std::printf("Cylinder force postprocess, paper formula\n");
    std::printf("force patch   = %s\n", cyl.name.c_str());
    std::printf("force faces   = %d\n", cyl.nFaces);
    std::printf("force area    = %.12e\n", cyl.area);
    std::printf("rho, mu       = %.12e  %.12e\n", par.rho, mu);
    std::printf("Ubar, D, H    = %.12e  %.12e  %.12e\n", (4.0 / 9.0) * par.Umean, par.pipeDiameter, 0.41);
    std::printf("coeff denom   = rho*Ubar^2*D*H = %.12e\n", cyl.denom);
    std::printf("FD pressure   = %.12e\n", cyl.FDp);
    std::printf("FD viscous    = %.12e\n", cyl.FDv);
    std::printf("FD total      = %.12e\n", cyl.FDp + cyl.FDv);
    std::printf("FL pressure   = %.12e\n", cyl.FLp);
    std::printf("FL viscous    = %.12e\n", cyl.FLv);
    std::printf("FL total      = %.12e\n", cyl.FLp + cyl.FLv);
    std::printf("CD            = %.12e\n", cyl.CD);
    std::printf("CL            = %.12e\n", cyl.CL);
    std::printf("wall dn min/max = %.12e / %.12e\n", cyl.minDn, cyl.maxDn);
    std::printf("max|dvt/dn|   = %.12e\n", cyl.maxDvt);
    std::printf("------------------------------------------------------------\n");
    std::printf("Cylinder force postprocess, vector wall-shear traction\n");
    std::printf("force patch   = %s\n", cyl.name.c_str());
    std::printf("force faces   = %d\n", cyl.nFaces);
    std::printf("force area    = %.12e\n", cyl.area);
    std::printf("rho, mu       = %.12e  %.12e\n", par.rho, mu);
    std::printf("Ubar, D, H    = %.12e  %.12e  %.12e\n", (4.0 / 9.0) * par.Umean, par.pipeDiameter, 0.41);
    std::printf("coeff denom   = rho*Ubar^2*D*H = %.12e\n", cyl.denom);
    std::printf("Fp vector     = [%.12e, %.12e, %.12e]\n", cyl.Fp[0], cyl.Fp[1], cyl.Fp[2]);
    std::printf("Fv vector     = [%.12e, %.12e, %.12e]\n", cyl.Fv[0], cyl.Fv[1], cyl.Fv[2]);
    std::printf("F  vector     = [%.12e, %.12e, %.12e]\n", cyl.F[0], cyl.F[1], cyl.F[2]);
    std::printf("C  vector     = [%.12e, %.12e, %.12e]\n", cyl.Cv[0], cyl.Cv[1], cyl.Cv[2]);
    std::printf("CD_vector     = %.12e\n", cyl.Cv[0]);
    std::printf("CL_y_vector   = %.12e\n", cyl.Cv[1]);
    std::printf("CL_z_vector   = %.12e\n", cyl.Cv[2]);
    std::printf("wall dn min/max = %.12e / %.12e\n", cyl.vminDn, cyl.vmaxDn);
    std::printf("max|Ut|       = %.12e\n", cyl.maxUt);
    std::printf("max shear mag = %.12e\n", cyl.maxShear);
  } else {
    std::printf("Cylinder force postprocess skipped: patch_3_0 not found.\n");
  }
  if (par.forceEnable) {
    std::printf("------------------------------------------------------------\n");
    if (pf.valid) {
      std::printf("Patch force postprocess, raw Cartesian wall traction\n");
      std::printf("force patch       = %s\n", par.forcePatchName.c_str());
      std::printf("force faces       = %d\n", pf.n_faces);
      std::printf("force area        = %.12e\n", pf.area);
      std::printf("normalSign        = %d\n", par.forceNormalSign);
      std::printf("rho, mu           = %.12e  %.12e\n", par.rho, mu);
      std::printf("pressureForce     = [%.12e, %.12e, %.12e]\n", pf.Fp[0], pf.Fp[1], pf.Fp[2]);
      std::printf("viscousForce      = [%.12e, %.12e, %.12e]\n", pf.Fv[0], pf.Fv[1], pf.Fv[2]);
      std::printf("totalForce        = [%.12e, %.12e, %.12e]\n", pf.F[0], pf.F[1], pf.F[2]);
      const char* ax[3] = {"x", "y", "z"};
      for (int d = 0; d < 3; ++d) std::printf("pressureForce_%s   = %.12e\n", ax[d], pf.Fp[d]);
      for (int d = 0; d < 3; ++d) std::printf("viscousForce_%s    = %.12e\n", ax[d], pf.Fv[d]);
      for (int d = 0; d < 3; ++d) std::printf("totalForce_%s      = %.12e\n", ax[d], pf.F[d]);
      std::printf("wall dn min/max   = %.12e / %.12e\n", pf.min_wall_distance, pf.max_wall_distance);
      std::printf("max|Ut|           = %.12e\n", pf.max_ut);
      std::printf("max shear mag     = %.12e\n", pf.max_shear_mag);
    } else {
      std::printf("Patch force postprocess requested but skipped. Check forcePatch.\n");
      std::printf("requested patch  = %s\n", par.forcePatchName.c_str());
      std::printf("forceUref        = %.12e\n", par.forceUref);
      std::printf("forceAreaRef     = %.12e\n", par.forceAreaRef);
    }
  }
  std::printf("last bicgstab it = [%d %d %d]\n", last.its_u, last.its_v, last.its_w);
  std::printf("last pcg it   = %d\n", last.its_p_last);
  std::printf("setup time    : %.6e s\n", tSetup);
  std::printf("device time   : %.6e s\n", gpuSeconds);
  std::printf("solve loop wall: %.6e s\n", loopWall);
  std::printf("cell-iters/s  : %.6e\n", loopWall > 0 ? (double)mesh.nCells * stepConverged / loopWall : 0.0);
  if (par.write_vtu) {
    std::string vtu = par.outPrefix + "_final.vtu";
    try {
      write_vtu_fields(mesh, vtu, u, v, w, p, divCorr, par.vtuBinary != 0);
    } catch (const std::exception& e) {
      die(e.what());
    }
    std::printf("Wrote VTU         : %s\n", vtu.c_str());
  }
  std::ofstream so(par.outPrefix + "_summary.txt");
  so << std::setprecision(16);
  so << "points " << mesh.points.size() << "\nfaces " << mesh.nFaces << "\ninternalFaces " << mesh.nInternalFaces
     << "\ncells " << mesh.nCells << "\n";
  so << "maxNonOrthDeg " << mesh.maxNonOrthDeg << "\nmu " << mu << "\n";
  so << "steps " << stepConverged << "\nmassRes " << last.mass_res << "\n";
  so << "maxAbsU " << umax << "\nmaxAbsV " << vmaxf << "\nmaxAbsW " << wmaxf << "\nmaxAbsP " << pmax << "\n";
  so << "lastBiCGSTABU " << last.its_u << "\nlastBiCGSTABV " << last.its_v << "\nlastBiCGSTABW " << last.its_w
     << "\nlastPCG " << last.its_p_last << "\n";
  if (cyl.valid) {
    so << "cylinderForcePatch " << cyl.name << "\ncylinderForceFaces " << cyl.nFaces << "\ncylinderForceArea "
       << cyl.area << "\nforceUbar " << (4.0 / 9.0) * par.Umean << "\nforceD " << par.pipeDiameter << "\nforceH "
       << 0.41 << "\nforceCoeffDenom " << cyl.denom << "\nFDPressure " << cyl.FDp << "\nFDViscous " << cyl.FDv
       << "\nFDTotal " << cyl.FDp + cyl.FDv << "\nFLPressure " << cyl.FLp << "\nFLViscous " << cyl.FLv
       << "\nFLTotal " << cyl.FLp + cyl.FLv << "\nCD " << cyl.CD << "\nCL " << cyl.CL << "\nwallDnMin "
       << cyl.minDn << "\nwallDnMax " << cyl.maxDn << "\nmaxAbsDvtDn " << cyl.maxDvt << "\n";
    so << "CDVector " << cyl.Cv[0] << "\nCLyVector " << cyl.Cv[1] << "\nCLzVector " << cyl.Cv[2] << "\n";
    so << "FxPressureVector " << cyl.Fp[0] << "\nFyPressureVector " << cyl.Fp[1] << "\nFzPressureVector " << cyl.Fp[2]
       << "\nFxViscousVector " << cyl.Fv[0] << "\nFyViscousVector " << cyl.Fv[1] << "\nFzViscousVector "
       << cyl.Fv[2] << "\nFxTotalVector " << cyl.F[0] << "\nFyTotalVector " << cyl.F[1] << "\nFzTotalVector "
       << cyl.F[2] << "\n";
  }
  if (pf.valid) {
    so << "patchForcePatch " << par.forcePatchName << "\npatchForceFaces " << pf.n_faces << "\npatchForceArea "
       << pf.area << "\npatchForceNormalSign " << par.forceNormalSign << "\n";
    so << "pressureForce_x " << pf.Fp[0] << "\npressureForce_y " << pf.Fp[1] << "\npressureForce_z " << pf.Fp[2] << "\n";
    so << "viscousForce_x " << pf.Fv[0] << "\nviscousForce_y " << pf.Fv[1] << "\nviscousForce_z " << pf.Fv[2] << "\n";
    so << "totalForce_x " << pf.F[0] << "\ntotalForce_y " << pf.F[1] << "\ntotalForce_z " << pf.F[2] << "\n";
  }
  so.close();
  anb_destroy(ctx);
  return 0;
}
