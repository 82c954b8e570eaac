// Read-only views of a context's device data for entry points implemented outside anb_api.cu.
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

struct anb_ctx;

namespace anb {

// Inputs of the patch-force integral for one patch (boundary-face range [b0, b1)).
struct ForceView {
  DMesh dm;
  int b0 = 0, b1 = 0;
  double mu = 0.0;
  const double* bA = nullptr;   // boundary face areas
  const double* bN = nullptr;   // boundary face unit normals (3 per face)
  const double* U = nullptr;    // velocity (3 * nCells)
  const double* P = nullptr;    // pressure
  cudaStream_t stream = nullptr;
  int device = 0;
};

// Returns false when `patch` is not a patch of the context's mesh.
bool context_force_view(const anb_ctx* c, int patch, ForceView* v);
void context_set_error(anb_ctx* c, const char* msg);
// Places the allocation-free force integral's static scratch and kernel on `device` (the current
// device); returns 0 on success.  Called by anb_create.
int nalloc_prepare_device(int device);

}  // namespace anb
