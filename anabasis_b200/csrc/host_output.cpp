// VTU writers (polyhedron cells).  write_vtu is the reference's ASCII writer, main.cu:975-983:
// same XML layout, the same point/connectivity/face streams and the same number formatting
// (%.15g for Float64).  write_vtu_appended writes the same arrays as raw little-endian binary in
// one appended block (exact values, no text formatting), for large meshes.
#include "host_output.hpp"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <vector>

namespace anb {

namespace {
struct Out {
  std::FILE* fp;
  std::vector<char> buf;
  size_t n = 0;
  explicit Out(std::FILE* f) : fp(f), buf(1 << 20) {}
  ~Out() { flush(); }
  void flush() {
    if (n) std::fwrite(buf.data(), 1, n, fp);
    n = 0;
  }
  void put(const char* s) {
    while (*s) {
      if (n == buf.size()) flush();
      buf[n++] = *s++;
    }
  }
  void num(double v) {
    char t[40];
    std::snprintf(t, sizeof t, "%.15g", v);
    put(t);
  }
  void num(long long v) {
    char t[32];
    std::snprintf(t, sizeof t, "%lld", v);
    put(t);
  }
};
}  // namespace

namespace {

// Polyhedron cell streams of the VTU (main.cu:975-983): per cell its unique points in face order
// (faces in cell-face order, neighbour-side faces reversed), the face stream
// [nFaces, n0, p.., n1, p.., ...] and the running offsets of both.
struct CellStreams {
  std::vector<long long> conn, offsets, faces, faceOff;
};

CellStreams cell_streams(const HostMesh& m) {
  const int nC = m.nCells;
  CellStreams s;
  s.offsets.resize(nC);
  s.faceOff.resize(nC);
  long long connCount = 0, faceCount = 0;
  std::vector<int> allPts, uniq;
  std::vector<std::vector<int>> cellFacePts;
  for (int c = 0; c < nC; ++c) {
    const int j0 = m.cellFaceOff[c], j1 = m.cellFaceOff[c + 1];
    cellFacePts.assign(j1 - j0, {});
    allPts.clear();
    for (int j = j0; j < j1; ++j) {
      const int f = m.cellFaces[j];
      auto& fp = cellFacePts[j - j0];
      fp.assign(m.facePts.begin() + m.faceOff[f], m.facePts.begin() + m.faceOff[f + 1]);
      if (m.cellFaceOri[j] < 0) std::reverse(fp.begin(), fp.end());
      allPts.insert(allPts.end(), fp.begin(), fp.end());
    }
    uniq.clear();
    for (int p : allPts)
      if (std::find(uniq.begin(), uniq.end(), p) == uniq.end()) uniq.push_back(p);
    for (int p : uniq) s.conn.push_back(p);
    connCount += (long long)uniq.size();
    s.offsets[c] = connCount;
    s.faces.push_back((long long)(j1 - j0));
    for (const auto& fp : cellFacePts) {
      s.faces.push_back((long long)fp.size());
      for (int p : fp) s.faces.push_back(p);
    }
    faceCount += 1;
    for (const auto& fp : cellFacePts) faceCount += 1 + (long long)fp.size();
    s.faceOff[c] = faceCount;
  }
  return s;
}

}  // namespace

void write_vtu(const HostMesh& m, const std::string& filename, const std::vector<std::string>& names,
               const std::vector<const double*>& data, const char* vecName, const double* const* vec) {
  const int nPts = m.nPoints(), nC = m.nCells;
  const CellStreams cs = cell_streams(m);
  const auto& conn = cs.conn;
  const auto& offsets = cs.offsets;
  const auto& faces = cs.faces;
  const auto& faceOff = cs.faceOff;
  std::FILE* fp = std::fopen(filename.c_str(), "w");
  if (!fp) throw std::runtime_error("Could not open " + filename + " for writing");
  {
    Out o(fp);
    o.put("<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" byte_order=\"LittleEndian\">\n  <UnstructuredGrid>\n    <Piece NumberOfPoints=\"");
    o.num((long long)nPts);
    o.put("\" NumberOfCells=\"");
    o.num((long long)nC);
    o.put("\">\n      <Points>\n        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (const auto& p : m.points) {
      o.put("          ");
      o.num(p[0]); o.put(" "); o.num(p[1]); o.put(" "); o.num(p[2]); o.put("\n");
    }
    o.put("        </DataArray>\n      </Points>\n      <Cells>\n        <DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n          ");
    for (long long v : conn) { o.num(v); o.put(" "); }
    o.put("\n        </DataArray>\n        <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n          ");
    for (long long v : offsets) { o.num(v); o.put(" "); }
    o.put("\n        </DataArray>\n        <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n          ");
    for (int c = 0; c < nC; ++c) o.put("42 ");
    o.put("\n        </DataArray>\n        <DataArray type=\"Int64\" Name=\"faces\" format=\"ascii\">\n          ");
    for (long long v : faces) { o.num(v); o.put(" "); }
    o.put("\n        </DataArray>\n        <DataArray type=\"Int64\" Name=\"faceoffsets\" format=\"ascii\">\n          ");
    for (long long v : faceOff) { o.num(v); o.put(" "); }
    o.put("\n        </DataArray>\n      </Cells>\n      <CellData>\n");
    if (vec) {
      o.put("        <DataArray type=\"Float64\" Name=\"");
      o.put(vecName);
      o.put("\" NumberOfComponents=\"3\" format=\"ascii\">\n");
      for (int c = 0; c < nC; ++c) {
        o.put("          ");
        o.num(vec[0][c]); o.put(" "); o.num(vec[1][c]); o.put(" "); o.num(vec[2][c]); o.put("\n");
      }
      o.put("        </DataArray>\n");
    }
    for (size_t k = 0; k < names.size(); ++k) {
      o.put("        <DataArray type=\"Float64\" Name=\"");
      o.put(names[k].c_str());
      o.put("\" NumberOfComponents=\"1\" format=\"ascii\">\n");
      for (int c = 0; c < nC; ++c) {
        o.put("          ");
        o.num(data[k][c]);
        o.put("\n");
      }
      o.put("        </DataArray>\n");
    }
    o.put("      </CellData>\n    </Piece>\n  </UnstructuredGrid>\n</VTKFile>\n");
  }
  std::fclose(fp);
}

void write_vtu_appended(const HostMesh& m, const std::string& filename, const std::vector<std::string>& names,
                        const std::vector<const double*>& data, const char* vecName, const double* const* vec) {
  const int nPts = m.nPoints(), nC = m.nCells;
  const CellStreams cs = cell_streams(m);
  // the arrays of the appended block, in order; each is stored as a UInt64 byte count + raw data
  struct Arr {
    std::string type, name;
    int comps;
    uint64_t bytes;
  };
  std::vector<Arr> arrs;
  arrs.push_back({"Float64", "", 3, 24ull * nPts});
  arrs.push_back({"Int64", "connectivity", 1, 8ull * cs.conn.size()});
  arrs.push_back({"Int64", "offsets", 1, 8ull * cs.offsets.size()});
  arrs.push_back({"UInt8", "types", 1, (uint64_t)nC});
  arrs.push_back({"Int64", "faces", 1, 8ull * cs.faces.size()});
  arrs.push_back({"Int64", "faceoffsets", 1, 8ull * cs.faceOff.size()});
  if (vec) arrs.push_back({"Float64", vecName, 3, 24ull * nC});
  for (const auto& nm : names) arrs.push_back({"Float64", nm, 1, 8ull * nC});
  std::vector<uint64_t> off(arrs.size());
  uint64_t cur = 0;
  for (size_t k = 0; k < arrs.size(); ++k) {
    off[k] = cur;
    cur += 8 + arrs[k].bytes;
  }
  std::FILE* fp = std::fopen(filename.c_str(), "wb");
  if (!fp) throw std::runtime_error("Could not open " + filename + " for writing");
  auto decl = [&](size_t k, const char* indent) {
    const Arr& a = arrs[k];
    std::fprintf(fp, "%s<DataArray type=\"%s\"", indent, a.type.c_str());
    if (!a.name.empty()) std::fprintf(fp, " Name=\"%s\"", a.name.c_str());
    if (a.comps > 1 || k == 0) std::fprintf(fp, " NumberOfComponents=\"%d\"", a.comps);
    std::fprintf(fp, " format=\"appended\" offset=\"%llu\"/>\n", (unsigned long long)off[k]);
  };
  std::fprintf(fp, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" "
                   "byte_order=\"LittleEndian\" header_type=\"UInt64\">\n  <UnstructuredGrid>\n"
                   "    <Piece NumberOfPoints=\"%d\" NumberOfCells=\"%d\">\n      <Points>\n", nPts, nC);
  decl(0, "        ");
  std::fprintf(fp, "      </Points>\n      <Cells>\n");
  for (size_t k = 1; k <= 5; ++k) decl(k, "        ");
  std::fprintf(fp, "      </Cells>\n      <CellData>\n");
  for (size_t k = 6; k < arrs.size(); ++k) decl(k, "        ");
  std::fprintf(fp, "      </CellData>\n    </Piece>\n  </UnstructuredGrid>\n  <AppendedData encoding=\"raw\">\n_");
  auto block = [&](const void* p, uint64_t bytes) {
    std::fwrite(&bytes, sizeof bytes, 1, fp);
    if (bytes) std::fwrite(p, 1, bytes, fp);
  };
  {
    std::vector<double> pts(3 * (size_t)nPts);
    for (int i = 0; i < nPts; ++i)
      for (int q = 0; q < 3; ++q) pts[3 * (size_t)i + q] = m.points[i][q];
    block(pts.data(), arrs[0].bytes);
  }
  block(cs.conn.data(), arrs[1].bytes);
  block(cs.offsets.data(), arrs[2].bytes);
  {
    std::vector<uint8_t> types(nC, 42);
    block(types.data(), arrs[3].bytes);
  }
  block(cs.faces.data(), arrs[4].bytes);
  block(cs.faceOff.data(), arrs[5].bytes);
  size_t k = 6;
  if (vec) {
    std::vector<double> v(3 * (size_t)nC);
    for (int c = 0; c < nC; ++c)
      for (int q = 0; q < 3; ++q) v[3 * (size_t)c + q] = vec[q][c];
    block(v.data(), arrs[k++].bytes);
  }
  for (size_t j = 0; j < names.size(); ++j) block(data[j], arrs[k++].bytes);
  std::fprintf(fp, "\n  </AppendedData>\n</VTKFile>\n");
  if (std::fclose(fp) != 0) throw std::runtime_error("Could not write " + filename);
}

}  // namespace anb
