// Device layout of a polyMesh for the SIMPLE kernels (built on the host once per mesh).
//
// Cells are renumbered by reverse Cuthill-McKee; every internal face is re-oriented so that its
// owner is the lower new cell index and faces are sorted by (owner, neighbour).  The discrete
// operators of the reference (apps/generic_simple_v1/src/main.cu:1403-1967) are invariant under
// that re-orientation (lambda -> 1-lambda, n -> -n, d -> -d), so every cell quantity is unchanged
// and face fluxes only change sign; the output path maps them back.
//
// Matrix off-diagonals use sliced ELLPACK with slice height 32 (SELL-32): entry k of row r lives
// at sliceOff[r/32] + 32*k + r%32, so a warp reads 32 consecutive column indices / values per
// step.  The diagonal is a separate dense vector.  The same pattern serves the momentum and the
// pressure matrices (the reference's two patterns coincide without the pressure anchor,
// main.cu:1315-1374 with usePressureAnchor=false at main.cu:3294).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "host_mesh.hpp"

namespace anb {

constexpr int kSlice = 32;

enum FaceFlag : uint8_t {
  kFaceAsm = 1,      // n.d > 1e-14: momentum / pressure assembly (main.cu:1727,1826,1916,1947)
  kFaceNonOrth = 2,  // |n.d| > 1e-30: non-orthogonal flux (main.cu:1560,1583,1648)
};

struct Layout {
  int nCells = 0, nInternal = 0, nBoundary = 0, nPatches = 0;
  // wall seconds of the build: adjacency, LSQ moments, RCM, face order + coefficients, SELL pattern,
  // boundary faces + cell data
  double seconds[6] = {0, 0, 0, 0, 0, 0};
  std::vector<int> new2old, old2new;  // cells

  // SELL-32 off-diagonal pattern
  int nSlices = 0;
  std::vector<int> sliceOff;   // nSlices+1 (entries)
  std::vector<int> rowLen;     // nCells
  std::vector<int> col;        // padded entries hold the row itself
  std::vector<int> slotFace;   // internal face (new index) of the entry, -1 on padding
  int maxRowLen = 0;

  // internal faces in new order
  std::vector<int> fOwner, fNeigh;     // new cell ids, owner < neigh
  std::vector<int> fOrig;              // original face index
  std::vector<uint8_t> fFlip;          // 1 if the original owner is the new neighbour
  std::vector<double> fLam;            // clamped interpolation weight toward the neighbour
  std::vector<double> fG;              // A / max(n.d, 1e-30)
  std::vector<double> fT;              // 3*nInternal: S - (A/n.d) d
  std::vector<double> fD;              // 3*nInternal: cc_N - cc_P
  std::vector<uint8_t> fFlags;

  // boundary faces in input order (boundary index b <-> original face nInternal + b)
  std::vector<int> bOwner, bPatch;
  std::vector<double> bG, bT, bS;      // A/n.d_b, S - (A/n.d_b) d_b, S (3 per face)
  std::vector<uint8_t> bFlags;
  std::vector<int> cbOff, cbList;      // cell -> boundary faces

  // cells
  std::vector<double> vol, cc;         // cc: 3*nCells
  std::vector<double> minv;            // 6*nCells: xx, xy, xz, yy, yz, zz of the LSQ inverse
};

// Throws std::runtime_error when two internal faces join the same pair of cells (not supported).
// Distinct neighbours of every cell, ascending, in input numbering (cellNbrs, main.cu:595-596);
// throws when two internal faces join the same pair of cells.
void cell_adjacency(const HostMesh& m, std::vector<int>& off, std::vector<int>& adj);
// LSQ moment inverse (build_lsq_gradient_operator, main.cu:1169-1224), 6 per cell in input
// numbering, on the host.
std::vector<double> lsq_minv_host(const HostMesh& m, const std::vector<int>& off, const std::vector<int>& adj);
// The device layout from the mesh, its adjacency and its moment inverses (input numbering).
Layout build_layout(const HostMesh& m, const std::vector<int>& off, const std::vector<int>& adj,
                    const std::vector<double>& minvOrig);
// Same, with the adjacency and moments computed on the host.
Layout build_layout(const HostMesh& m);

// LSQ moment inverse of the scalar libraries (libpoisson/src/gradient.cu:21-83,
// libscalar/src/scalar_transport_library.cu:185-246): neighbours as in the SIMPLE operator,
// Dirichlet boundary faces at the face centre, every other boundary face as the pure-normal
// constraint r = max((x_f - x_P).n, 1e-30) n.  bDirichlet has one entry per boundary face (input
// order); the result is 6 per cell in the layout's cell order.
std::vector<double> scalar_lsq_minv(const HostMesh& m, const Layout& L, const std::vector<uint8_t>& bDirichlet);

// Reverse Cuthill-McKee order of an undirected graph in CSR form (new2old).
std::vector<int> rcm_order(int n, const std::vector<int>& adjOff, const std::vector<int>& adj);

}  // namespace anb
