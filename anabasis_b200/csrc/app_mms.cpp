// Drop-in replacements of the reference's manufactured-solution programs, built four times from
// this file (ANB_MMS_APP selects which):
//   1 anabasis_poisson_mms          apps/poisson_mms_lib/main.cu          (phi = sin sin sin)
//   2 anabasis_poisson_mms_neumann  apps/poisson_mms_neumann_lib/main.cu  (cos cos cos, all Neumann)
//   3 anabasis_poisson_mms_mixed    apps/poisson_mms_mixed_lib/main.cu    (cos cos cos, mixed BCs)
//   4 anabasis_scalar_mms           apps/scalar_mms_lib/main.cu           (convection-diffusion)
// Same flags, defaults, error messages and summary lines; the HYPRE/BoomerAMG flags are accepted
// and ignored (the solves are libanb.so's AMG-PCG and Jacobi-BiCGSTAB).  The exact fields are the
// analytic functions of the reference programs (libpoisson/include/mms.h and the programs).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/anb.h"
#include "host_mesh.hpp"

#ifndef ANB_MMS_APP
#define ANB_MMS_APP 1
#endif

using anb::HostMesh;
using anb::Vec3;

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

[[noreturn]] void die(const std::string& msg) {
  std::fprintf(stderr, "%s\n", msg.c_str());
  std::exit(1);
}

struct Params {
  std::string polyMeshDir = ANB_MMS_APP == 4 ? "/tmp/unitcube_hex_50mm/constant/polyMesh" : "./mesh/constant/polyMesh";
  int device = 0;
  int nNonOrthCorr = ANB_MMS_APP == 4 ? 0 : 10;
  int monitor = ANB_MMS_APP == 4 ? 0 : 1;
  int maxIter = 4000;
  double tol = ANB_MMS_APP == 1 ? 1e-12 : 1e-10;
  std::string gradScheme = "lsq", laplacianScheme = "nonorth";
  std::string dirichletPatchesCsv, neumannPatchesCsv;
  int useReferenceCell = ANB_MMS_APP == 2 ? 1 : 0;
  int referenceCell = 0;
  int referenceValueUserSet = 0;
  double referenceValue = 0.0;
  // scalar transport program
  double gamma = 0.1;
  std::string convectionScheme = "central", diffusionScheme = "orth";
  std::string transportMode = "convection_diffusion", bcMode = "dirichlet";
};

std::vector<std::string> split_csv(const std::string& s) {
  std::vector<std::string> out;
  std::stringstream ss(s);
  std::string item;
  while (std::getline(ss, item, ',')) {
    std::string t;
    for (char ch : item)
      if (ch != ' ' && ch != '\t' && ch != '\n' && ch != '\r') t.push_back(ch);
    if (!t.empty()) out.push_back(t);
  }
  return out;
}

void parse_args(int argc, char** argv, Params& p) {
  static const char* kIgnoredInt[] = {"-amg-maxit", "-amg-relax-type", "-amg-coarsen-type", "-amg-interp-type",
                                      "-amg-agg-levels", "-amg-pmax", "-amg-keep-transpose"};
  static const char* kIgnoredDbl[] = {"-amg-trunc-factor", "-amg-strong-threshold"};
  for (int i = 1; i < argc; ++i) {
    const std::string o = argv[i];
    auto need = [&]() {
      if (i + 1 >= argc) die("Missing value after " + o);
      return std::string(argv[++i]);
    };
    bool ignored = false;
    if (ANB_MMS_APP != 4) {
      for (const char* k : kIgnoredInt) ignored = ignored || o == k;
      for (const char* k : kIgnoredDbl) ignored = ignored || o == k;
    }
    if (ignored) {
      need();
    } else if (o == "-polyMeshDir") {
      p.polyMeshDir = need();
    } else if (o == "-device") {
      p.device = std::atoi(need().c_str());
    } else if (o == "-nNonOrthCorr") {
      p.nNonOrthCorr = std::atoi(need().c_str());
    } else if (o == "-monitor") {
      p.monitor = std::atoi(need().c_str());
    } else if (o == "-maxit") {
      p.maxIter = std::atoi(need().c_str());
    } else if (o == "-tol") {
      p.tol = std::atof(need().c_str());
    } else if (ANB_MMS_APP != 4 && o == "-grad-scheme") {
      p.gradScheme = need();
    } else if (ANB_MMS_APP != 4 && o == "-laplacian-scheme") {
      p.laplacianScheme = need();
    } else if ((ANB_MMS_APP == 1 || ANB_MMS_APP == 3 || ANB_MMS_APP == 4) && o == "-dirichlet-patches") {
      p.dirichletPatchesCsv = need();
    } else if (ANB_MMS_APP == 1 && o == "-neumann-patches") {
      p.neumannPatchesCsv = need();
    } else if ((ANB_MMS_APP == 1 || ANB_MMS_APP == 2) && o == "-use-reference-cell") {
      p.useReferenceCell = std::atoi(need().c_str());
    } else if ((ANB_MMS_APP == 1 || ANB_MMS_APP == 2) && o == "-reference-cell") {
      p.referenceCell = std::atoi(need().c_str());
    } else if ((ANB_MMS_APP == 1 || ANB_MMS_APP == 2) && o == "-reference-value") {
      p.referenceValue = std::atof(need().c_str());
      p.referenceValueUserSet = 1;
    } else if (ANB_MMS_APP == 4 && o == "-gamma") {
      p.gamma = std::atof(need().c_str());
    } else if (ANB_MMS_APP == 4 && o == "-convection-scheme") {
      p.convectionScheme = need();
    } else if (ANB_MMS_APP == 4 && o == "-diffusion-scheme") {
      p.diffusionScheme = need();
    } else if (ANB_MMS_APP == 4 && o == "-transport-mode") {
      p.transportMode = need();
    } else if (ANB_MMS_APP == 4 && o == "-bc-mode") {
      p.bcMode = need();
    } else {
      die("Unknown option: " + o);
    }
  }
}

// exact fields
double sin3(const Vec3& x) { return std::sin(kPi * x[0]) * std::sin(kPi * x[1]) * std::sin(kPi * x[2]); }
Vec3 grad_sin3(const Vec3& x) {
  const double sx = std::sin(kPi * x[0]), sy = std::sin(kPi * x[1]), sz = std::sin(kPi * x[2]);
  const double cx = std::cos(kPi * x[0]), cy = std::cos(kPi * x[1]), cz = std::cos(kPi * x[2]);
  return {kPi * cx * sy * sz, kPi * sx * cy * sz, kPi * sx * sy * cz};
}
double cos3(const Vec3& x) { return std::cos(kPi * x[0]) * std::cos(kPi * x[1]) * std::cos(kPi * x[2]); }
Vec3 grad_cos3(const Vec3& x) {
  const double sx = std::sin(kPi * x[0]), sy = std::sin(kPi * x[1]), sz = std::sin(kPi * x[2]);
  const double cx = std::cos(kPi * x[0]), cy = std::cos(kPi * x[1]), cz = std::cos(kPi * x[2]);
  return {-kPi * sx * cy * cz, -kPi * cx * sy * cz, -kPi * cx * cy * sz};
}
double dot(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
Vec3 velocity(const Vec3& x) { return {1.0 + x[1], 0.5 - x[0], 0.25}; }

double phi_exact(const Vec3& x) { return ANB_MMS_APP == 1 || ANB_MMS_APP == 4 ? sin3(x) : cos3(x); }
Vec3 grad_exact(const Vec3& x) { return ANB_MMS_APP == 1 || ANB_MMS_APP == 4 ? grad_sin3(x) : grad_cos3(x); }

struct Norms {
  double l1 = 0, l2 = 0, linf = 0, vmin = std::numeric_limits<double>::max(),
         vmax = -std::numeric_limits<double>::max(), mean = 0;
};

Norms norms(const HostMesh& m, const std::vector<double>& phi, double shift) {
  Norms n;
  double V = 0;
  for (int c = 0; c < m.nCells; ++c) {
    const double raw = phi[c] - phi_exact(m.cc[c]);
    const double e = std::fabs(raw - shift);
    V += m.vol[c];
    n.mean += m.vol[c] * raw;
    n.l1 += m.vol[c] * e;
    n.l2 += m.vol[c] * e * e;
    n.linf = std::max(n.linf, e);
    n.vmin = std::min(n.vmin, phi[c]);
    n.vmax = std::max(n.vmax, phi[c]);
  }
  V = std::max(V, 1e-30);
  n.l1 /= V;
  n.l2 = std::sqrt(n.l2 / V);
  n.mean /= V;
  return n;
}

}  // namespace

int main(int argc, char** argv) {
  Params par;
  parse_args(argc, argv, par);
  if (ANB_MMS_APP == 3 && par.dirichletPatchesCsv.empty())
    die("You must provide -dirichlet-patches patchA[,patchB,...]");
  if (cudaSetDevice(par.device) != cudaSuccess) die("CUDA ERROR: cannot select the device");
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, par.device) != cudaSuccess) die("CUDA ERROR: no device properties");
  std::printf("Running on GPU \"%s\" (cc %d.%d), total memory %.2f GiB\n", prop.name, prop.major, prop.minor,
              (double)prop.totalGlobalMem / (1024.0 * 1024.0 * 1024.0));
  std::printf("Reading mesh from %s\n", par.polyMeshDir.c_str());
  HostMesh mesh;
  try {
    mesh = anb::read_polymesh(par.polyMeshDir);
  } catch (const std::exception& e) {
    die(e.what());
  }
  std::printf("Mesh stats: cells=%d, faces=%d, internalFaces=%d, boundaryPatches=%zu, maxNonOrthDeg=%.3f\n",
              mesh.nCells, mesh.nFaces, mesh.nInternalFaces, mesh.patches.size(), mesh.maxNonOrthDeg);
  for (size_t i = 0; i < mesh.patches.size(); ++i) std::printf("  patch[%zu] = %s\n", i, mesh.patches[i].name.c_str());

  // boundary types per patch
  const auto dirList = split_csv(par.dirichletPatchesCsv);
  const auto neuList = split_csv(par.neumannPatchesCsv);
  const std::set<std::string> dirSet(dirList.begin(), dirList.end()), neuSet(neuList.begin(), neuList.end());
  if (ANB_MMS_APP == 3) {
    for (const auto& d : dirSet) {
      bool found = false;
      for (const auto& pt : mesh.patches) found = found || pt.name == d;
      if (!found) die("Dirichlet patch '" + d + "' not found in mesh");
    }
  }
  if (ANB_MMS_APP == 4) {
    if (par.transportMode != "diffusion_only" && par.transportMode != "convection_diffusion")
      die("Unsupported transportMode '" + par.transportMode + "'. Use convection_diffusion or diffusion_only.");
    if (par.bcMode != "dirichlet" && par.bcMode != "mixed")
      die("Unsupported bcMode '" + par.bcMode + "'. Use dirichlet or mixed.");
  }
  std::vector<int> bt(mesh.nFaces, ANB_SCALAR_DIRICHLET);
  std::vector<double> bv(mesh.nFaces, 0.0);
  for (const auto& pt : mesh.patches) {
    bool dirichlet = true;
    if (ANB_MMS_APP == 1) dirichlet = !neuSet.count(pt.name);
    if (ANB_MMS_APP == 2) dirichlet = false;
    if (ANB_MMS_APP == 3) dirichlet = dirSet.count(pt.name) > 0;
    if (ANB_MMS_APP == 4) dirichlet = par.bcMode == "dirichlet" || dirSet.count(pt.name) > 0;
    for (int f = pt.start; f < pt.start + pt.nFaces; ++f) {
      bt[f] = dirichlet ? ANB_SCALAR_DIRICHLET : ANB_SCALAR_NEUMANN;
      bv[f] = dirichlet ? phi_exact(mesh.xf[f]) : dot(grad_exact(mesh.xf[f]), mesh.nf[f]);
    }
  }
  if (ANB_MMS_APP == 3) {
    std::printf("Dirichlet patches: %s\n", par.dirichletPatchesCsv.c_str());
    std::printf("All remaining boundary patches are Neumann.\n");
  }

  // context
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
  anb_params prm;
  anb_default_params(&prm);
  prm.device = par.device;
  anb_ctx* ctx = nullptr;
  if (anb_create(&md, &prm, &ctx) != ANB_OK) die(std::string("anb_create: ") + anb_last_error(nullptr));

  std::vector<double> phi(mesh.nCells, 0.0), src(mesh.nCells);
  anb_solve_info info{};
  int rc;
  if (ANB_MMS_APP != 4) {
    if (par.gradScheme != "lsq") die("Only gradScheme=lsq is implemented in this build.");
    if (par.laplacianScheme != "orth" && par.laplacianScheme != "nonorth")
      die("Use laplacianScheme=orth or laplacianScheme=nonorth.");
    for (int c = 0; c < mesh.nCells; ++c) src[c] = 3.0 * kPi * kPi * phi_exact(mesh.cc[c]);
    if (ANB_MMS_APP == 2) {
      double s = 0, V = 0;
      for (int c = 0; c < mesh.nCells; ++c) {
        s += src[c] * mesh.vol[c];
        V += mesh.vol[c];
      }
      const double mean = s / std::max(V, 1e-30);
      for (double& x : src) x -= mean;  // discrete compatibility of the pure-Neumann problem
      std::printf("Discrete source mean removed: %.12e\n", mean);
      if (par.useReferenceCell) {
        if (par.referenceCell < 0 || par.referenceCell >= mesh.nCells)
          die("referenceCell " + std::to_string(par.referenceCell) + " out of range [0," +
              std::to_string(mesh.nCells) + ")");
        if (!par.referenceValueUserSet) par.referenceValue = phi_exact(mesh.cc[par.referenceCell]);
      }
    }
    rc = anb_scalar_elliptic_solve(ctx, nullptr, src.data(), bt.data(), bv.data(), par.laplacianScheme == "nonorth",
                                   par.nNonOrthCorr, par.useReferenceCell, par.referenceCell, par.referenceValue,
                                   par.tol, 0.0, par.maxIter, phi.data(), &info);
  } else {
    const bool diffOnly = par.transportMode == "diffusion_only";
    std::vector<double> flux(mesh.nFaces, 0.0), gam(mesh.nFaces, par.gamma), sp(mesh.nCells, 0.0);
    for (int f = 0; f < mesh.nFaces && !diffOnly; ++f) flux[f] = dot(velocity(mesh.xf[f]), mesh.Sf[f]);
    for (int c = 0; c < mesh.nCells; ++c) {
      const double diff = 3.0 * par.gamma * kPi * kPi * sin3(mesh.cc[c]);
      src[c] = diffOnly ? diff : dot(velocity(mesh.cc[c]), grad_sin3(mesh.cc[c])) + diff;
    }
    const bool upwind = par.convectionScheme == "upwind" || par.convectionScheme == "upwind1";
    rc = anb_scalar_transport_solve(ctx, flux.data(), gam.data(), src.data(), sp.data(), bt.data(), bv.data(),
                                    upwind ? ANB_CONVECTION_UPWIND : ANB_CONVECTION_CENTRAL,
                                    par.diffusionScheme == "nonorth", par.nNonOrthCorr, par.tol, 0.0, par.maxIter,
                                    nullptr, phi.data(), &info);
  }
  if (rc != ANB_OK && rc != ANB_NOT_CONVERGED) die(std::string("solve: ") + anb_last_error(ctx));
  if (rc == ANB_NOT_CONVERGED) std::fprintf(stderr, "WARNING: linear solve did not converge\n");
  anb_destroy(ctx);

  const Norms n = norms(mesh, phi, 0.0);
  if (ANB_MMS_APP == 4) {
    std::printf("\n=== Scalar convection-diffusion MMS summary ===\n");
    std::printf("convectionScheme: %s\n", par.convectionScheme.c_str());
    std::printf("diffusionScheme : %s\n", par.diffusionScheme.c_str());
    std::printf("nNonOrthCorr    : %d\n", par.nNonOrthCorr);
    std::printf("gamma           : %.6e\n", par.gamma);
    std::printf("transportMode   : %s\n", par.transportMode.c_str());
    std::printf("bcMode          : %s\n", par.bcMode.c_str());
    if (par.bcMode == "mixed") std::printf("dirichletPatches: %s\n", par.dirichletPatchesCsv.c_str());
    std::printf("last solver its : %d\n", info.iterations);
    std::printf("last relRes     : %.12e\n", info.final_rel_res);
  } else {
    static const char* kTitle[] = {"", "Poisson MMS", "Poisson Neumann MMS", "Poisson Mixed-BC MMS"};
    std::printf("\n=== %s summary ===\n", kTitle[ANB_MMS_APP]);
    std::printf("gradScheme      : %s\n", par.gradScheme.c_str());
    std::printf("laplacianScheme : %s\n", par.laplacianScheme.c_str());
    std::printf("nNonOrthCorr    : %d\n", par.nNonOrthCorr);
    std::printf("last hypreIts   : %d\n", info.iterations);
    std::printf("last relRes     : %.12e\n", info.final_rel_res);
    if (ANB_MMS_APP == 2 && par.useReferenceCell) {
      std::printf("referenceCell   : %d\n", par.referenceCell);
      std::printf("referenceValue  : %.12e\n", par.referenceValue);
    }
    if (ANB_MMS_APP == 3) std::printf("Dirichlet patches: %s\n", par.dirichletPatchesCsv.c_str());
  }
  std::printf("solution min/max: %.12e  %.12e\n", n.vmin, n.vmax);
  std::printf("L1 error        : %.12e\n", n.l1);
  std::printf("L2 error        : %.12e\n", n.l2);
  std::printf("Linf error      : %.12e\n", n.linf);
  if (ANB_MMS_APP == 2) {
    const Norms s = norms(mesh, phi, n.mean);
    std::printf("mean err shift  : %.12e\n", n.mean);
    std::printf("L1 shifted      : %.12e\n", s.l1);
    std::printf("L2 shifted      : %.12e\n", s.l2);
    std::printf("Linf shifted    : %.12e\n", s.linf);
  }
  return 0;
}
