// Mesh set-up on the device (setup_gpu.cu): geometry, LSQ moment inverse, slot-ordered face records.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "device.cuh"
#include "host_mesh.hpp"

namespace anb {

// Cell volumes and centroids, face centres, areas, unit normals and area vectors of m (topology
// finalized) on the device, bit-identical to compute_geometry, downloaded into m.  Throws with
// compute_geometry's messages.  Returns false (m untouched) when a cell has more distinct points
// than the device kernel holds; the caller then uses compute_geometry.
bool compute_geometry_gpu(HostMesh& m, cudaStream_t s);

// lsq_minv_host on the device (bit-identical): 6 per cell in input numbering.
std::vector<double> lsq_minv_gpu(const HostMesh& m, const std::vector<int>& off, const std::vector<int>& adj,
                                 cudaStream_t s);

// slotGeom (8 arrays of nE doubles) and slotFlags from the face records through slotFace
// (all device pointers), zero on padding slots.
void build_slot_geometry(size_t nE, const int* slotFace, const FaceRec* face, const uint8_t* fFlags, double* slotGeom,
                         uint8_t* slotFlags, cudaStream_t s);

}  // namespace anb
