// Host-side polyMesh container, ASCII reader/writer, finite-volume geometry and the
// synthetic channel-mesh generator.
//
// The reader and the geometry follow apps/generic_simple_v1/src/main.cu:532-599 of the
// reference (read_openfoam_polymesh): the same list grammar, the same error messages, and
// the same floating-point operation order, so that cell centres, volumes, face centres,
// normals and areas come out bit-identical to the reference's own host code.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace anb {

using Vec3 = std::array<double, 3>;

struct PatchInfo {
  std::string name;
  std::string type;
  int start = 0;
  int nFaces = 0;
};

// Topology in OpenFOAM order plus the derived geometry (filled by compute_geometry).
struct HostMesh {
  std::vector<Vec3> points;
  std::vector<int> faceOff;   // nFaces+1
  std::vector<int> facePts;   // CSR point labels
  std::vector<int> owner;     // nFaces
  std::vector<int> neigh;     // nInternalFaces
  std::vector<PatchInfo> patches;
  std::vector<int> bPatch;    // nFaces, 1-based patch id for boundary faces, 0 for internal
  int nFaces = 0, nInternalFaces = 0, nCells = 0;

  // geometry (main.cu:591-597)
  std::vector<Vec3> cc, xf, nf, Sf;
  std::vector<double> vol, Af;
  double maxNonOrthDeg = 0.0;

  // cell -> faces in the reference's order: faces owned by the cell (ascending), then faces
  // where the cell is the neighbour (ascending)  (main.cu:588-590)
  std::vector<int> cellFaceOff, cellFaces;
  std::vector<signed char> cellFaceOri;

  int nPoints() const { return (int)points.size(); }
};

// Throws std::runtime_error with the reference's messages ("Could not open <file>",
// "Could not locate top-level OpenFOAM list", "Failed to match parentheses",
// "Malformed faces list").
HostMesh read_polymesh(const std::string& polyMeshDir);
void write_polymesh(const HostMesh& m, const std::string& polyMeshDir);

// Builds bPatch and the cell->face lists, then the geometry.  Throws
// "Non-positive cell volume at cell N" / "Degenerate face area at face N".
void finalize_topology(HostMesh& m);
void compute_geometry(HostMesh& m, int nThreads = 0);
// Largest angle between an internal face normal and its cell-centre vector, in degrees (main.cu:598).
void max_nonorth_deg(HostMesh& m);

struct ChannelSpec {
  int nx = 40, ny = 20, nz = 20;
  double Lx = 2.5, Ly = 0.41, Lz = 0.41;
  double jitter = 0.0;          // fraction of local spacing, uniform in [-j, j]
  uint64_t seed = 0;
  bool obstacle = false;        // remove cells whose (unjittered) centre lies in the block
  double ox0 = 0.45, ox1 = 0.55, oy0 = 0.15, oy1 = 0.25;
  bool tets = false;            // split every hex into 6 tets (Kuhn split)
};

// Channel box meshed by hexes (optionally jittered, with a removed obstacle block, or split
// into tets).  Patches: patch_0_0 (4 walls), patch_1_0 (inlet x=0), patch_2_0 (outlet x=Lx),
// patch_3_0 (obstacle, only when present).  Faces are in OpenFOAM order: internal faces in
// upper-triangular order, then boundary faces grouped by patch.
HostMesh make_channel_mesh(const ChannelSpec& s);

}  // namespace anb
