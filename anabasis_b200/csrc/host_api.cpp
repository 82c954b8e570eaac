// C ABI of the host front end (include/anb_host.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/anb_host.h"
#include "host_case.hpp"
#include "host_mesh.hpp"
#include "host_output.hpp"

struct anb_hmesh {
  anb::HostMesh m;
  bool geom = false;
};

namespace {
int set_err(char* buf, int len, const char* msg) {
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", msg);
  return 1;
}
void ensure_geom(anb_hmesh* h) {
  if (!h->geom) {
    anb::compute_geometry(h->m);
    h->geom = true;
  }
}
}  // namespace

extern "C" {

int anb_mesh_read_polymesh(const char* dir, anb_hmesh** out, char* eb, int el) {
  try {
    auto* h = new anb_hmesh();
    try {
      h->m = anb::read_polymesh(dir);
    } catch (...) {
      delete h;
      throw;
    }
    h->geom = true;
    *out = h;
    return 0;
  } catch (const std::exception& e) {
    return set_err(eb, el, e.what());
  }
}

int anb_mesh_make_channel(int nx, int ny, int nz, double lx, double ly, double lz, double jitter,
                          unsigned long long seed, int obstacle, int tets, anb_hmesh** out, char* eb, int el) {
  try {
    anb::ChannelSpec s;
    s.nx = nx; s.ny = ny; s.nz = nz;
    s.Lx = lx; s.Ly = ly; s.Lz = lz;
    s.jitter = jitter;
    s.seed = seed;
    s.obstacle = obstacle != 0;
    s.tets = tets != 0;
    auto* h = new anb_hmesh();
    try {
      h->m = anb::make_channel_mesh(s);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
    return 0;
  } catch (const std::exception& e) {
    return set_err(eb, el, e.what());
  }
}

int anb_mesh_write_polymesh(const anb_hmesh* h, const char* dir, char* eb, int el) {
  try {
    anb::write_polymesh(h->m, dir);
    return 0;
  } catch (const std::exception& e) {
    return set_err(eb, el, e.what());
  }
}

void anb_mesh_free(anb_hmesh* h) { delete h; }

void anb_mesh_sizes(const anb_hmesh* h, int* s) {
  const auto& m = h->m;
  s[0] = m.nPoints();
  s[1] = (int)m.faceOff.size() - 1;
  s[2] = (int)m.facePts.size();
  s[3] = (int)m.neigh.size();
  s[4] = m.nCells;
  s[5] = (int)m.patches.size();
}

void anb_mesh_topology(const anb_hmesh* h, double* pts, int* fo, int* fp, int* own, int* nei, int* ps, int* pn) {
  const auto& m = h->m;
  if (pts)
    for (int i = 0; i < m.nPoints(); ++i)
      for (int k = 0; k < 3; ++k) pts[3 * i + k] = m.points[i][k];
  if (fo) std::memcpy(fo, m.faceOff.data(), sizeof(int) * m.faceOff.size());
  if (fp) std::memcpy(fp, m.facePts.data(), sizeof(int) * m.facePts.size());
  if (own) std::memcpy(own, m.owner.data(), sizeof(int) * m.owner.size());
  if (nei && !m.neigh.empty()) std::memcpy(nei, m.neigh.data(), sizeof(int) * m.neigh.size());
  for (size_t k = 0; k < m.patches.size(); ++k) {
    if (ps) ps[k] = m.patches[k].start;
    if (pn) pn[k] = m.patches[k].nFaces;
  }
}

const char* anb_mesh_patch_name(const anb_hmesh* h, int p) {
  if (p < 0 || p >= (int)h->m.patches.size()) return "";
  return h->m.patches[p].name.c_str();
}

int anb_mesh_geometry(anb_hmesh* h, double* cc, double* vol, double* xf, double* nf, double* sf, double* af,
                      double* mx, char* eb, int el) {
  try {
    ensure_geom(h);
    const auto& m = h->m;
    for (int c = 0; c < m.nCells; ++c) {
      if (cc) for (int k = 0; k < 3; ++k) cc[3 * c + k] = m.cc[c][k];
      if (vol) vol[c] = m.vol[c];
    }
    for (int f = 0; f < m.nFaces; ++f) {
      for (int k = 0; k < 3; ++k) {
        if (xf) xf[3 * f + k] = m.xf[f][k];
        if (nf) nf[3 * f + k] = m.nf[f][k];
        if (sf) sf[3 * f + k] = m.Sf[f][k];
      }
      if (af) af[f] = m.Af[f];
    }
    if (mx) *mx = m.maxNonOrthDeg;
    return 0;
  } catch (const std::exception& e) {
    return set_err(eb, el, e.what());
  }
}

int anb_bc_evaluate(anb_hmesh* h, const char* path, int* tu, int* tv, int* tw, int* tp, double* u, double* v,
                    double* w, double* p, double* table, char* eb, int el) {
  try {
    ensure_geom(h);
    const auto& m = h->m;
    anb::BCConfig cfg = anb::load_bc_config(path);
    std::vector<std::string> names;
    for (const auto& pi : m.patches) names.push_back(pi.name);
    anb::validate_bc_config(cfg, names);
    auto geom = anb::build_patch_geometry(m);
    anb::FaceBC bc = anb::evaluate_face_bc(m, geom, cfg);
    const int nP = (int)m.patches.size();
    for (int k = 0; k < nP; ++k) {
      tu[k] = bc.typeU[k];
      tv[k] = bc.typeV[k];
      tw[k] = bc.typeW[k];
      tp[k] = bc.typeP[k];
      if (table) {
        double* t = table + 10 * k;
        t[0] = geom[k].totalArea;
        for (int q = 0; q < 3; ++q) {
          t[1 + q] = geom[k].centroid[q];
          t[4 + q] = geom[k].averageNormal[q];
        }
        t[7] = geom[k].planarity;
        t[8] = geom[k].nFaces;
        t[9] = std::sqrt(geom[k].sumSf[0] * geom[k].sumSf[0] + geom[k].sumSf[1] * geom[k].sumSf[1] +
                         geom[k].sumSf[2] * geom[k].sumSf[2]);
      }
    }
    std::memcpy(u, bc.u.data(), sizeof(double) * m.nFaces);
    std::memcpy(v, bc.v.data(), sizeof(double) * m.nFaces);
    std::memcpy(w, bc.w.data(), sizeof(double) * m.nFaces);
    std::memcpy(p, bc.p.data(), sizeof(double) * m.nFaces);
    return 0;
  } catch (const std::exception& e) {
    return set_err(eb, el, e.what());
  }
}

int anb_expand_case_args(int argc, const char* const* argv, char* out, int outlen, char* eb, int el) {
  try {
    std::vector<std::string> a(argv, argv + argc);
    auto r = anb::expand_case_config_args(a);
    size_t need = 0;
    for (const auto& s : r) need += s.size() + 1;
    if ((int)need > outlen) {
      set_err(eb, el, "output buffer too small");
      return -1;
    }
    size_t o = 0;
    for (const auto& s : r) {
      std::memcpy(out + o, s.c_str(), s.size() + 1);
      o += s.size() + 1;
    }
    return (int)r.size();
  } catch (const std::exception& e) {
    set_err(eb, el, e.what());
    return -1;
  }
}

int anb_write_vtu(anb_hmesh* h, const char* fn, const double* u, const double* v, const double* w, const double* p,
                  const double* divCorr, char* eb, int el) {
  try {
    ensure_geom(h);
    const auto& m = h->m;
    std::vector<double> umag(m.nCells);
    for (int c = 0; c < m.nCells; ++c) umag[c] = std::sqrt(u[c] * u[c] + v[c] * v[c] + w[c] * w[c]);
    const double* vec[3] = {u, v, w};
    anb::write_vtu(m, fn, {"p", "umag", "cell_volume", "divCorr"}, {p, umag.data(), m.vol.data(), divCorr}, "U", vec);
    return 0;
  } catch (const std::exception& e) {
    return set_err(eb, el, e.what());
  }
}

int anb_write_vtu_binary(anb_hmesh* h, const char* fn, const double* u, const double* v, const double* w,
                         const double* p, const double* divCorr, char* eb, int el) {
  try {
    ensure_geom(h);
    const auto& m = h->m;
    std::vector<double> umag(m.nCells);
    for (int c = 0; c < m.nCells; ++c) umag[c] = std::sqrt(u[c] * u[c] + v[c] * v[c] + w[c] * w[c]);
    const double* vec[3] = {u, v, w};
    anb::write_vtu_appended(m, fn, {"p", "umag", "cell_volume", "divCorr"}, {p, umag.data(), m.vol.data(), divCorr},
                            "U", vec);
    return 0;
  } catch (const std::exception& e) {
    return set_err(eb, el, e.what());
  }
}

}  // extern "C"
