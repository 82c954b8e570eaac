// Runtime configuration front end: `.case` files, command-line flags, `.bc` boundary-condition
// files, patch geometry summaries and per-face boundary values.
//
// Behaviour follows the reference's drop-in interface:
//   .case expansion      apps/generic_simple_v1/src/main.cu:162-331 (expand_case_config_args)
//   flag parsing         main.cu:333-401 (parse_args), defaults main.cu:73-103 (Params)
//   .bc grammar          apps/generic_simple_v1/src/bc_runtime_config.cu:83-230
//   BC kinds             apps/generic_simple_v1/src/bc_specs.{h,cu}
//   patch table          apps/generic_simple_v1/src/patch_geometry.cu:84-140
//   face values          apps/generic_simple_v1/src/velocity_bc_eval.cu:42-290
#pragma once

#include <array>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "host_mesh.hpp"

namespace anb {

// Error carrying the process exit code the reference would have produced.
struct CliError : std::runtime_error {
  int code;
  CliError(const std::string& m, int c = 1) : std::runtime_error(m), code(c) {}
};

struct Params {
  std::string polyMeshDir = "/tmp/meshCase/constant/polyMesh";
  std::string outPrefix = "pipe_poiseuille_gpu";
  double rho = 1.0, mu = 0.05, Re = 1.0, Umean = 1.0, CFL = 1.0;
  bool muExplicit = false;
  double pipeDiameter = 0.05, pipeLength = 0.50;
  std::string wallPatchName = "patch_0_0", inletPatchName = "patch_1_0", outletPatchName = "patch_2_0";
  std::string bcConfigPath;
  int device = 0, velRestart = 40, velMaxit = 100, monitor = 1, write_vtu = 1;
  int vtuBinary = 0;             // anbVtuFormat binary: appended raw VTU instead of the reference's ASCII
  int nVelNonOrthCorr = 0, nNonOrthCorr = 2, nPressureCorr = 0, nsteps = 1000, printEvery = 25, writeEvery = 0;
  double velTol = 1e-10, velRelTol = 0.0, corrTol = 1e-12, tolMass = 1e-10, tolVel = 1e-10;
  double uRelax = 0.7, pRelax = 1.0;
  int p_use_amg = 1, pMaxit = 4000, pAmgMaxit = 1, pAmgRelaxType = 18, pAmgCoarsenType = 8, pAmgInterpType = 3,
      pAmgAggLevels = 1, pAmgAggInterpType = 4, pAmgPmax = 4, pAmgKeepTranspose = 0;
  double pTol = 1e-10, pRelTol = 0.0, pAmgTruncFactor = 0.2;
  int profileSteps = 0;
  int pAmgRebuildEvery = 1;
  int pAmgSetupScope = 0;
  int forceEnable = 0;
  std::string forcePatchName;
  int forceNormalSign = -1;
  std::array<double, 3> forceDragDir{{1.0, 0.0, 0.0}};
  std::array<double, 3> forceLiftDir{{0.0, 1.0, 0.0}};
  std::array<double, 3> forceSpanDir{{0.0, 0.0, 1.0}};
  double forceUref = -1.0, forceAreaRef = -1.0;
  // Extensions (keys the reference rejects): precision "fp64" (0) or "mixed" (1).
  int precision = 0;
};

// Expands `-case-config <file>` into flags; inline velocity/pressure lines are written to
// `<case>.generated.bc`.  Throws std::runtime_error with the reference's messages.
std::vector<std::string> expand_case_config_args(const std::vector<std::string>& argv);
// Throws CliError on a missing flag value / bad vector / bad setup scope.
void parse_args(const std::vector<std::string>& argv, Params& par);

enum class VelKind { WallNoSlip, FixedUniformVector, ZeroGradient, FixedNormalSpeed, FixedFlowRate, ParabolicBoxInlet };
enum class PresKind { FixedValue, ZeroGradient, Open };
enum class NormalMode { AveragePatchNormal, LocalFaceNormal };

struct VelocitySpec {
  std::string patch;
  VelKind kind = VelKind::ZeroGradient;
  std::array<double, 3> vec{{0, 0, 0}};
  double normalSpeed = 0.0, flowRate = 0.0;
  NormalMode mode = NormalMode::AveragePatchNormal;
  double H = 1.0, Umax = 1.0;
  int coordA = 1, coordB = 2;
};
struct PressureSpec {
  std::string patch;
  PresKind kind = PresKind::ZeroGradient;
  double value = 0.0;
};
struct BCConfig {
  std::vector<VelocitySpec> vel;
  std::vector<PressureSpec> pres;
};

BCConfig load_bc_config(const std::string& path);
void validate_bc_config(const BCConfig& cfg, const std::vector<std::string>& patchNames);
std::vector<std::string> duplicate_velocity_patches(const BCConfig& cfg);
std::vector<std::string> duplicate_pressure_patches(const BCConfig& cfg);
bool pressure_reference_required(const BCConfig& cfg);

struct PatchGeom {
  int index = -1;
  std::string name;
  int nFaces = 0;
  double totalArea = 0.0;
  Vec3 centroid{{0, 0, 0}}, sumSf{{0, 0, 0}}, averageNormal{{0, 0, 0}};
  double planarity = 0.0;
  Vec3 tangent1{{0, 0, 0}}, tangent2{{0, 0, 0}};
};
std::vector<PatchGeom> build_patch_geometry(const HostMesh& m);

// Per-patch BC type (1 = Dirichlet, 0 = Neumann) for U,V,W,P and per-face values
// (arrays of nFaces; internal entries stay 0).
struct FaceBC {
  std::vector<int> typeU, typeV, typeW, typeP;
  std::vector<double> u, v, w, p;
};
FaceBC evaluate_face_bc(const HostMesh& m, const std::vector<PatchGeom>& geom, const BCConfig& cfg);

}  // namespace anb
