// ASCII VTU writer (polyhedron cells), main.cu:975-983 of the reference: same XML layout, the
// same point/connectivity/face streams and the same number formatting (%.15g for Float64).
#include "host_output.hpp"

#include <cmath>
#include <cstdio>
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

void write_vtu(const HostMesh& m, const std::string& filename, const std::vector<std::string>& names,
               const std::vector<const double*>& data, const char* vecName, const double* const* vec) {
  const int nPts = m.nPoints(), nC = m.nCells;
  std::vector<long long> conn, offsets(nC), faces, faceOff(nC);
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
    for (int p : uniq) conn.push_back(p);
    connCount += (long long)uniq.size();
    offsets[c] = connCount;
    faces.push_back((long long)(j1 - j0));
    for (const auto& fp : cellFacePts) {
      faces.push_back((long long)fp.size());
      for (int p : fp) faces.push_back(p);
    }
    faceCount += 1;
    for (const auto& fp : cellFacePts) faceCount += 1 + (long long)fp.size();
    faceOff[c] = faceCount;
  }
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

}  // namespace anb
