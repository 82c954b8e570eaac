// VTU writers of cell data on polyhedral cells: ASCII (reference main.cu:975-983) and appended binary.
#pragma once

#include <algorithm>
#include <string>
#include <vector>

#include "host_mesh.hpp"

namespace anb {

// Writes points, polyhedron cells (type 42) and cell data: the vector field `vecName`
// (vec[0..2], may be NULL) followed by the scalar fields.
void write_vtu(const HostMesh& m, const std::string& filename, const std::vector<std::string>& names,
               const std::vector<const double*>& data, const char* vecName, const double* const* vec);
// The same arrays as raw little-endian binary in one <AppendedData encoding="raw"> block
// (header_type UInt64): exact values, written without text formatting.
void write_vtu_appended(const HostMesh& m, const std::string& filename, const std::vector<std::string>& names,
                        const std::vector<const double*>& data, const char* vecName, const double* const* vec);

}  // namespace anb
