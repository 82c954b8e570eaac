// Runtime configuration front end (.case / flags / .bc / patch table / face BC values).
#include "host_case.hpp"

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <unordered_map>
#include <unordered_set>

namespace anb {
namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}
std::string strip_hash(const std::string& s) {
  size_t h = s.find('#');
  return h == std::string::npos ? s : s.substr(0, h);
}
std::vector<std::string> tokens(const std::string& line) {
  std::istringstream is(line);
  std::vector<std::string> t;
  for (std::string x; is >> x;) t.push_back(x);
  return t;
}

// .case key -> flag (main.cu:182-251) plus this build's extension keys (prefix "anb").
const std::map<std::string, std::string>& case_keys() {
  static const std::map<std::string, std::string> k = {
      {"polyMeshDir", "-polyMeshDir"}, {"outPrefix", "-out-prefix"}, {"rho", "-rho"}, {"mu", "-mu"},
      {"re", "-re"}, {"Re", "-re"}, {"uMean", "-uMean"}, {"Umean", "-uMean"}, {"pipeD", "-pipeD"},
      {"pipeL", "-pipeL"}, {"wallPatch", "-wall-patch"}, {"inletPatch", "-inlet-patch"},
      {"outletPatch", "-outlet-patch"}, {"bcConfig", "-bc-config"}, {"device", "-device"}, {"cfl", "-cfl"},
      {"CFL", "-cfl"}, {"nsteps", "-nsteps"}, {"printEvery", "-print-every"}, {"writeVtu", "-write-vtu"},
      {"writeEvery", "-write-every"}, {"monitor", "-monitor"}, {"velRestart", "-vel-restart"},
      {"velMaxit", "-vel-maxit"}, {"velTol", "-vel-tol"}, {"velRelTol", "-vel-reltol"},
      {"nVelNonOrthCorr", "-nVelNonOrthCorr"}, {"nNonOrthCorr", "-nNonOrthCorr"},
      {"nPressureCorr", "-nPressureCorr"}, {"uRelax", "-u-relax"}, {"pRelax", "-p-relax"},
      {"corrTol", "-corrTol"}, {"tolMass", "-tolMass"}, {"tolVel", "-tolVel"}, {"pUseAmg", "-p-use-amg"},
      {"pMaxit", "-p-maxit"}, {"pTol", "-p-tol"}, {"pRelTol", "-p-reltol"},
      {"pAmgSetupScope", "-p-amg-setup-scope"}, {"pAmgMaxit", "-p-amg-maxit"},
      {"pAmgCoarsenType", "-p-amg-coarsen-type"}, {"pAmgInterpType", "-p-amg-interp-type"},
      {"pAmgAggLevels", "-p-amg-agg-levels"}, {"pAmgAggInterpType", "-p-amg-agg-interp-type"},
      {"pAmgRelaxType", "-p-amg-relax-type"}, {"pAmgPmax", "-p-amg-pmax"},
      {"pAmgTruncFactor", "-p-amg-trunc-factor"}, {"pAmgKeepTranspose", "-p-amg-keep-transpose"},
      {"pAmgRebuildEvery", "-p-amg-rebuild-every"}, {"forceEnable", "-force-enable"},
      {"forcePatch", "-force-patch"}, {"forceNormalSign", "-force-normal-sign"},
      {"forceDragDir", "-force-drag-dir"}, {"forceLiftDir", "-force-lift-dir"},
      {"forceSpanDir", "-force-span-dir"}, {"forceUref", "-force-uref"}, {"forceAreaRef", "-force-area-ref"},
      {"profileSteps", "-profile-steps"}, {"assemblyBackend", "-assembly-backend"},
      {"anbPrecision", "-anb-precision"}, {"anbVtuFormat", "-anb-vtu-format"}};
  return k;
}

std::array<double, 3> parse_vec3_arg(const std::string& raw, const char* opt) {
  std::string t = raw;
  for (char& c : t)
    if (c == ',' || c == ';' || c == ':') c = ' ';
  std::istringstream is(t);
  std::array<double, 3> v{{0, 0, 0}};
  if (!(is >> v[0] >> v[1] >> v[2]))
    throw CliError(std::string("Could not parse ") + opt + " value '" + raw + "'. Expected x,y,z", 1);
  return v;
}

[[noreturn]] void bc_fail(const std::string& path, int line, const std::string& msg) {
  throw std::runtime_error("BC config parse error in '" + path + "' at line " + std::to_string(line) + ": " + msg);
}

double bc_double(const std::string& tok, const std::string& path, int line, const std::string& what) {
  // std::stod semantics: leading blanks allowed, whole token consumed, range errors rejected
  const char* s = tok.c_str();
  char* end = nullptr;
  errno = 0;
  double v = std::strtod(s, &end);
  if (end == s || errno == ERANGE || (size_t)(end - s) != tok.size())
    bc_fail(path, line, "invalid numeric token for " + what + ": '" + tok + "'");
  return v;
}

NormalMode bc_mode(const std::string& tok, const std::string& path, int line) {
  if (tok == "average_patch_normal") return NormalMode::AveragePatchNormal;
  if (tok == "local_face_normal") return NormalMode::LocalFaceNormal;
  bc_fail(path, line, "normal mode must be 'average_patch_normal' or 'local_face_normal', got '" + tok + "'");
}

int bc_coord(const std::string& tok, const std::string& path, int line) {
  if (tok == "x" || tok == "X" || tok == "0") return 0;
  if (tok == "y" || tok == "Y" || tok == "1") return 1;
  if (tok == "z" || tok == "Z" || tok == "2") return 2;
  bc_fail(path, line, "coordinate must be x/y/z or 0/1/2, got '" + tok + "'");
}

inline double dot3(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline Vec3 cross3(const Vec3& a, const Vec3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline Vec3 normalize3(const Vec3& a) {
  double n = std::sqrt(dot3(a, a));
  if (n <= 1.0e-30) return {0, 0, 0};
  return {a[0] / n, a[1] / n, a[2] / n};
}
Vec3 normalized_or_throw(const Vec3& a, const std::string& what) {
  double n = std::sqrt(std::max(dot3(a, a), 0.0));
  if (n <= 1.0e-30) throw std::runtime_error("Cannot normalize vector for " + what);
  return {a[0] / n, a[1] / n, a[2] / n};
}
Vec3 choose_normal(const VelocitySpec& s, const PatchGeom& p, const Vec3& faceNormal) {
  if (s.mode == NormalMode::AveragePatchNormal)
    return normalized_or_throw(p.averageNormal, "AveragePatchNormal on patch '" + p.name + "'");
  return normalized_or_throw(faceNormal, "LocalFaceNormal on patch '" + p.name + "'");
}

Vec3 eval_velocity(const VelocitySpec& s, const PatchGeom& p, const Vec3& x, const Vec3& fn) {
  switch (s.kind) {
    case VelKind::WallNoSlip:
    case VelKind::ZeroGradient:
      return {0, 0, 0};
    case VelKind::FixedUniformVector:
      return s.vec;
    case VelKind::ParabolicBoxInlet: {
      const double H = s.H, Umax = s.Umax;
      if (H <= 0.0) throw std::runtime_error("ParabolicBoxInlet has non-positive H on patch '" + s.patch + "'");
      const int ia = s.coordA, ib = s.coordB;
      if (ia < 0 || ia > 2 || ib < 0 || ib > 2 || ia == ib)
        throw std::runtime_error("ParabolicBoxInlet has invalid coordinates on patch '" + s.patch + "'");
      auto clampH = [H](double v) { return v < 0.0 ? 0.0 : (v > H ? H : v); };
      const double a = clampH(x[ia]), b = clampH(x[ib]);
      const double H2 = H * H, H4 = H2 * H2;
      const double mag = 16.0 * Umax * a * b * (H - a) * (H - b) / H4;
      const Vec3 n = choose_normal(s, p, fn);
      return {-mag * n[0], -mag * n[1], -mag * n[2]};
    }
    case VelKind::FixedNormalSpeed:
    case VelKind::FixedFlowRate: {
      if (s.kind == VelKind::FixedFlowRate && s.mode == NormalMode::AveragePatchNormal && p.planarity < 0.98)
        throw std::runtime_error(
            "FixedFlowRate with AveragePatchNormal requires an approximately planar patch. Patch '" + p.name +
            "' has planarity = " + std::to_string(p.planarity) + ". Use LocalFaceNormal instead.");
      double un;
      if (s.kind == VelKind::FixedNormalSpeed) un = s.normalSpeed;
      else {
        if (p.totalArea <= 1.0e-30)
          throw std::runtime_error("Patch '" + p.name + "' has near-zero area for FixedFlowRate");
        un = s.flowRate / p.totalArea;
      }
      const Vec3 n = choose_normal(s, p, fn);
      return {un * n[0], un * n[1], un * n[2]};
    }
  }
  throw std::runtime_error("Unhandled VelocityBCType");
}

}  // namespace

std::vector<std::string> expand_case_config_args(const std::vector<std::string>& argv) {
  std::string casePath;
  for (size_t i = 1; i < argv.size(); ++i) {
    if (argv[i] == "-case-config") {
      if (i + 1 >= argv.size()) throw std::runtime_error("Missing value after -case-config");
      casePath = argv[i + 1];
      break;
    }
  }
  if (casePath.empty()) return argv;
  std::ifstream in(casePath);
  if (!in) throw std::runtime_error("Could not open case config file: " + casePath);
  std::vector<std::string> out{argv.empty() ? std::string("anabasis_simple") : argv[0]};
  std::vector<std::string> bcLines;
  bool explicitBC = false;
  std::string raw;
  int lineNo = 0;
  while (std::getline(in, raw)) {
    ++lineNo;
    const std::string line = trim(strip_hash(raw));
    if (line.empty()) continue;
    auto tok = tokens(line);
    if (tok.empty()) continue;
    if (tok[0] == "velocity" || tok[0] == "pressure") {
      bcLines.push_back(line);
      continue;
    }
    if (tok.size() != 2) {
      std::ostringstream o;
      o << "Case config parse error in '" << casePath << "' at line " << lineNo
        << ": expected '<key> <value>' or a velocity/pressure BC line";
      throw std::runtime_error(o.str());
    }
    auto it = case_keys().find(tok[0]);
    if (it == case_keys().end()) {
      std::ostringstream o;
      o << "Case config parse error in '" << casePath << "' at line " << lineNo << ": unknown key '" << tok[0]
        << "'";
      throw std::runtime_error(o.str());
    }
    if (tok[0] == "bcConfig") explicitBC = true;
    out.push_back(it->second);
    out.push_back(tok[1]);
  }
  if (!bcLines.empty() && explicitBC)
    throw std::runtime_error("Case config cannot contain both bcConfig and inline velocity/pressure BC lines");
  if (!bcLines.empty()) {
    const std::string gen = casePath + ".generated.bc";
    std::ofstream bo(gen);
    if (!bo) throw std::runtime_error("Could not write generated BC file: " + gen);
    bo << "# Auto-generated from " << casePath << "\n";
    for (const auto& l : bcLines) bo << l << "\n";
    out.push_back("-bc-config");
    out.push_back(gen);
  }
  for (size_t i = 1; i < argv.size(); ++i) {
    if (argv[i] == "-case-config") {
      ++i;
      continue;
    }
    out.push_back(argv[i]);
  }
  return out;
}

void parse_args(const std::vector<std::string>& a, Params& par) {
  const int argc = (int)a.size();
  for (int i = 1; i < argc; ++i) {
    auto need = [&](const std::string& opt) {
      if (i + 1 >= argc) throw CliError("Missing value after " + opt, 1);
    };
    const std::string& o = a[i];
    auto D = [&](double& x) { need(o); x = std::atof(a[++i].c_str()); };
    auto I = [&](int& x) { need(o); x = std::atoi(a[++i].c_str()); };
    auto S = [&](std::string& x) { need(o); x = a[++i]; };
    if (o == "-polyMeshDir") S(par.polyMeshDir);
    else if (o == "-out-prefix") S(par.outPrefix);
    else if (o == "-rho") D(par.rho);
    else if (o == "-mu") { D(par.mu); par.muExplicit = true; }
    else if (o == "-re") D(par.Re);
    else if (o == "-uMean" || o == "-lidU") D(par.Umean);
    else if (o == "-pipeD") D(par.pipeDiameter);
    else if (o == "-pipeL") D(par.pipeLength);
    else if (o == "-wall-patch") S(par.wallPatchName);
    else if (o == "-inlet-patch" || o == "-lid-patch") S(par.inletPatchName);
    else if (o == "-outlet-patch") S(par.outletPatchName);
    else if (o == "-bc-config") S(par.bcConfigPath);
    else if (o == "-force-enable") I(par.forceEnable);
    else if (o == "-force-patch") S(par.forcePatchName);
    else if (o == "-force-normal-sign") I(par.forceNormalSign);
    else if (o == "-force-drag-dir") { need(o); par.forceDragDir = parse_vec3_arg(a[++i], "-force-drag-dir"); }
    else if (o == "-force-lift-dir") { need(o); par.forceLiftDir = parse_vec3_arg(a[++i], "-force-lift-dir"); }
    else if (o == "-force-span-dir") { need(o); par.forceSpanDir = parse_vec3_arg(a[++i], "-force-span-dir"); }
    else if (o == "-force-uref") D(par.forceUref);
    else if (o == "-force-area-ref") D(par.forceAreaRef);
    else if (o == "-cfl") D(par.CFL);
    else if (o == "-device") I(par.device);
    else if (o == "-vel-restart") I(par.velRestart);
    else if (o == "-vel-maxit") I(par.velMaxit);
    else if (o == "-vel-tol") D(par.velTol);
    else if (o == "-vel-reltol") D(par.velRelTol);
    else if (o == "-nVelNonOrthCorr") I(par.nVelNonOrthCorr);
    else if (o == "-nNonOrthCorr") I(par.nNonOrthCorr);
    else if (o == "-nPressureCorr") I(par.nPressureCorr);
    else if (o == "-u-relax") D(par.uRelax);
    else if (o == "-p-relax") D(par.pRelax);
    else if (o == "-corrTol") D(par.corrTol);
    else if (o == "-monitor") I(par.monitor);
    else if (o == "-write-vtu") I(par.write_vtu);
    else if (o == "-nsteps") I(par.nsteps);
    else if (o == "-print-every") I(par.printEvery);
    else if (o == "-write-every") I(par.writeEvery);
    else if (o == "-tolMass") D(par.tolMass);
    else if (o == "-tolVel") D(par.tolVel);
    else if (o == "-p-use-amg") I(par.p_use_amg);
    else if (o == "-p-maxit") I(par.pMaxit);
    else if (o == "-p-tol") D(par.pTol);
    else if (o == "-p-reltol") D(par.pRelTol);
    else if (o == "-p-amg-maxit") I(par.pAmgMaxit);
    else if (o == "-p-amg-relax-type") I(par.pAmgRelaxType);
    else if (o == "-p-amg-coarsen-type") I(par.pAmgCoarsenType);
    else if (o == "-p-amg-interp-type") I(par.pAmgInterpType);
    else if (o == "-p-amg-agg-levels") I(par.pAmgAggLevels);
    else if (o == "-p-amg-agg-interp-type") I(par.pAmgAggInterpType);
    else if (o == "-p-amg-pmax") I(par.pAmgPmax);
    else if (o == "-p-amg-trunc-factor") D(par.pAmgTruncFactor);
    else if (o == "-p-amg-keep-transpose") I(par.pAmgKeepTranspose);
    else if (o == "-profile-steps") I(par.profileSteps);
    else if (o == "-p-amg-rebuild-every") I(par.pAmgRebuildEvery);
    else if (o == "-p-amg-setup-scope") {
      need(o);
      std::string v = a[++i];
      if (v == "outer") par.pAmgSetupScope = 0;
      else if (v == "pressure" || v == "solve") par.pAmgSetupScope = 1;
      else throw CliError("Unknown -p-amg-setup-scope '" + v + "'. Use outer or pressure.", 1);
    } else if (o == "-anb-precision") {
      need(o);
      std::string v = a[++i];
      if (v == "fp64" || v == "plain") par.precision = 0;
      else if (v == "mixed") par.precision = 1;
      else throw CliError("Unknown -anb-precision '" + v + "'. Use fp64 or mixed.", 1);
    } else if (o == "-anb-vtu-format") {
      need(o);
      std::string v = a[++i];
      if (v == "ascii") par.vtuBinary = 0;
      else if (v == "binary" || v == "appended") par.vtuBinary = 1;
      else throw CliError("Unknown -anb-vtu-format '" + v + "'. Use ascii or binary.", 1);
    }
  }
}

BCConfig load_bc_config(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("Could not open BC config file: " + path);
  BCConfig cfg;
  std::string raw;
  int ln = 0;
  while (std::getline(in, raw)) {
    ++ln;
    const std::string line = trim(strip_hash(raw));
    if (line.empty()) continue;
    auto t = tokens(line);
    if (t.empty()) continue;
    if (t[0] == "velocity") {
      if (t.size() < 3) bc_fail(path, ln, "velocity line must be: velocity <patch> <type> ...");
      VelocitySpec s;
      s.patch = t[1];
      const std::string& type = t[2];
      if (type == "wall_noslip") {
        if (t.size() != 3) bc_fail(path, ln, "wall_noslip takes no extra arguments");
        s.kind = VelKind::WallNoSlip;
      } else if (type == "zero_gradient") {
        if (t.size() != 3) bc_fail(path, ln, "zero_gradient takes no extra arguments");
        s.kind = VelKind::ZeroGradient;
      } else if (type == "fixed_uniform_vector") {
        if (t.size() != 6)
          bc_fail(path, ln, "fixed_uniform_vector syntax: velocity <patch> fixed_uniform_vector <ux> <uy> <uz>");
        s.kind = VelKind::FixedUniformVector;
        s.vec = {bc_double(t[3], path, ln, "ux"), bc_double(t[4], path, ln, "uy"), bc_double(t[5], path, ln, "uz")};
      } else if (type == "fixed_normal_speed") {
        if (t.size() != 4 && t.size() != 5)
          bc_fail(path, ln,
                  "fixed_normal_speed syntax: velocity <patch> fixed_normal_speed <value> "
                  "[average_patch_normal|local_face_normal]");
        s.kind = VelKind::FixedNormalSpeed;
        s.normalSpeed = bc_double(t[3], path, ln, "normal speed");
        s.mode = t.size() == 5 ? bc_mode(t[4], path, ln) : NormalMode::AveragePatchNormal;
      } else if (type == "fixed_flow_rate") {
        if (t.size() != 4 && t.size() != 5)
          bc_fail(path, ln,
                  "fixed_flow_rate syntax: velocity <patch> fixed_flow_rate <value> "
                  "[average_patch_normal|local_face_normal]");
        s.kind = VelKind::FixedFlowRate;
        s.flowRate = bc_double(t[3], path, ln, "flow rate");
        s.mode = t.size() == 5 ? bc_mode(t[4], path, ln) : NormalMode::AveragePatchNormal;
      } else if (type == "parabolic_box_inlet") {
        if (t.size() != 7 && t.size() != 8)
          bc_fail(path, ln,
                  "parabolic_box_inlet syntax: velocity <patch> parabolic_box_inlet <H> <Umax> <coord1> <coord2> "
                  "[average_patch_normal|local_face_normal]");
        s.kind = VelKind::ParabolicBoxInlet;
        s.H = bc_double(t[3], path, ln, "parabolic H");
        s.Umax = bc_double(t[4], path, ln, "parabolic Umax");
        s.coordA = bc_coord(t[5], path, ln);
        s.coordB = bc_coord(t[6], path, ln);
        if (s.coordA == s.coordB) bc_fail(path, ln, "parabolic_box_inlet requires two different transverse coordinates");
        s.mode = t.size() == 8 ? bc_mode(t[7], path, ln) : NormalMode::AveragePatchNormal;
      } else {
        bc_fail(path, ln, "unknown velocity BC type: '" + type + "'");
      }
      cfg.vel.push_back(s);
    } else if (t[0] == "pressure") {
      if (t.size() < 3) bc_fail(path, ln, "pressure line must be: pressure <patch> <type> ...");
      PressureSpec s;
      s.patch = t[1];
      const std::string& type = t[2];
      if (type == "zero_gradient") {
        if (t.size() != 3) bc_fail(path, ln, "zero_gradient takes no extra arguments");
        s.kind = PresKind::ZeroGradient;
      } else if (type == "open") {
        if (t.size() != 3) bc_fail(path, ln, "open takes no extra arguments");
        s.kind = PresKind::Open;
      } else if (type == "fixed_value") {
        if (t.size() != 4) bc_fail(path, ln, "fixed_value syntax: pressure <patch> fixed_value <value>");
        s.kind = PresKind::FixedValue;
        s.value = bc_double(t[3], path, ln, "pressure value");
      } else {
        bc_fail(path, ln, "unknown pressure BC type: '" + type + "'");
      }
      cfg.pres.push_back(s);
    } else {
      bc_fail(path, ln, "line must start with 'velocity' or 'pressure'");
    }
  }
  return cfg;
}

void validate_bc_config(const BCConfig& cfg, const std::vector<std::string>& names) {
  std::unordered_set<std::string> known(names.begin(), names.end());
  for (const auto& s : cfg.vel)
    if (!known.count(s.patch)) throw std::runtime_error("Velocity BC refers to unknown patch '" + s.patch + "'");
  for (const auto& s : cfg.pres)
    if (!known.count(s.patch)) throw std::runtime_error("Pressure BC refers to unknown patch '" + s.patch + "'");
}

template <class T>
static std::vector<std::string> dups(const std::vector<T>& v) {
  std::unordered_map<std::string, int> c;
  std::vector<std::string> d;
  for (const auto& s : v)
    if (++c[s.patch] == 2) d.push_back(s.patch);
  return d;
}
std::vector<std::string> duplicate_velocity_patches(const BCConfig& c) { return dups(c.vel); }
std::vector<std::string> duplicate_pressure_patches(const BCConfig& c) { return dups(c.pres); }

bool pressure_reference_required(const BCConfig& cfg) {
  for (const auto& s : cfg.pres)
    if (s.kind == PresKind::FixedValue) return false;
  return true;
}

std::vector<PatchGeom> build_patch_geometry(const HostMesh& m) {
  const int nP = (int)m.patches.size();
  std::vector<PatchGeom> out(nP);
  for (int p = 0; p < nP; ++p) {
    PatchGeom& g = out[p];
    g.index = p;
    g.name = m.patches[p].name;
    const int start = m.patches[p].start, count = m.patches[p].nFaces, end = start + count;
    if (count < 0 || start < m.nInternalFaces || end > m.nFaces)
      throw std::runtime_error("Invalid patch face range for patch '" + g.name + "'");
    g.nFaces = count;
    Vec3 acc{0, 0, 0}, sumSf{0, 0, 0};
    double area = 0.0;
    for (int f = start; f < end; ++f) {
      const double A = m.Af[f];
      area += A;
      acc = {acc[0] + A * m.xf[f][0], acc[1] + A * m.xf[f][1], acc[2] + A * m.xf[f][2]};
      sumSf = {sumSf[0] + m.Sf[f][0], sumSf[1] + m.Sf[f][1], sumSf[2] + m.Sf[f][2]};
    }
    g.totalArea = area;
    g.sumSf = sumSf;
    if (area > 1.0e-30) {
      const double r = 1.0 / area;
      g.centroid = {r * acc[0], r * acc[1], r * acc[2]};
    }
    const double sn = std::sqrt(dot3(sumSf, sumSf));
    g.averageNormal = normalize3(sumSf);
    g.planarity = area > 1.0e-30 ? sn / area : 0.0;
    const Vec3& n = g.averageNormal;
    if (std::sqrt(dot3(n, n)) > 0.0) {
      const double ax = std::fabs(n[0]), ay = std::fabs(n[1]), az = std::fabs(n[2]);
      Vec3 seed = (ax <= ay && ax <= az) ? Vec3{1, 0, 0} : ((ay <= ax && ay <= az) ? Vec3{0, 1, 0} : Vec3{0, 0, 1});
      g.tangent1 = normalize3(cross3(n, seed));
      g.tangent2 = normalize3(cross3(n, g.tangent1));
    } else {
      g.tangent1 = {1, 0, 0};
      g.tangent2 = {0, 1, 0};
    }
  }
  return out;
}

FaceBC evaluate_face_bc(const HostMesh& m, const std::vector<PatchGeom>& geom, const BCConfig& cfg) {
  const int nP = (int)m.patches.size();
  FaceBC bc;
  bc.typeU.assign(nP, 0);
  bc.typeV.assign(nP, 0);
  bc.typeW.assign(nP, 0);
  bc.typeP.assign(nP, 0);
  bc.u.assign(m.nFaces, 0.0);
  bc.v.assign(m.nFaces, 0.0);
  bc.w.assign(m.nFaces, 0.0);
  bc.p.assign(m.nFaces, 0.0);
  auto find = [&](const std::string& name) {
    for (int i = 0; i < nP; ++i)
      if (m.patches[i].name == name) return i;
    throw std::runtime_error("Patch '" + name + "' not found in LegacyBCMeshView");
  };
  auto findGeom = [&](const std::string& name) -> const PatchGeom& {
    for (const auto& g : geom)
      if (g.name == name) return g;
    throw std::runtime_error("Patch '" + name + "' not found in patch geometry table");
  };
  for (const auto& s : cfg.vel) {
    const int pi = find(s.patch);
    const PatchGeom& g = findGeom(s.patch);
    const int start = m.patches[pi].start, end = start + m.patches[pi].nFaces;
    if (s.kind == VelKind::ZeroGradient) {
      bc.typeU[pi] = bc.typeV[pi] = bc.typeW[pi] = 0;
      continue;
    }
    bc.typeU[pi] = bc.typeV[pi] = bc.typeW[pi] = 1;
    for (int f = start; f < end; ++f) {
      Vec3 U = eval_velocity(s, g, m.xf[f], m.nf[f]);
      bc.u[f] = U[0];
      bc.v[f] = U[1];
      bc.w[f] = U[2];
    }
  }
  for (const auto& s : cfg.pres) {
    const int pi = find(s.patch);
    const int start = m.patches[pi].start, end = start + m.patches[pi].nFaces;
    if (s.kind == PresKind::FixedValue) {
      bc.typeP[pi] = 1;
      for (int f = start; f < end; ++f) bc.p[f] = s.value;
    } else {
      bc.typeP[pi] = 0;
    }
  }
  return bc;
}

}  // namespace anb
