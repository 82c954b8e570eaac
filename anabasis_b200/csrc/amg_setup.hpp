// Host set-up of the aggregation AMG hierarchy for the pressure-correction matrix.
//
// Stands in for the BoomerAMG preconditioner the reference configures at
// apps/generic_simple_v1/src/main.cu:2242-2260.  The structure (aggregates, coarse patterns and
// Galerkin gather maps) is built once from the first assembled pressure matrix; every
// preconditioner rebuild afterwards (cadence pAmgRebuildEvery, main.cu:3409-3411) recomputes
// the coarse values on the device from the current fine matrix through the gather maps, so the
// hierarchy's values are stale between rebuilds exactly as the reference's are.
//
// Aggregation: two passes of pairwise matching per level (each row pairs with its strongest
// unmatched negative coupling, -a_ij >= beta * max_k(-a_ik)), giving aggregates of up to four
// rows; prolongation is piecewise constant, so A_c[I][J] = sum of a_ij over i in I, j in J.
#pragma once

#include <vector>

#include "layout.hpp"

namespace anb {

struct AmgLevelHost {
  int n = 0;
  // Off-diagonal pattern of this level (levels >= 1; level 0 uses the mesh layout's SELL-32
  // pattern).  Large coarse levels are SELL-32 like level 0 (sliceOff: slices of 32 rows, slot k of
  // row r at sliceOff[r/32] + 32k + r%32, padding slots point at the row itself with value 0) and
  // run the level-0 kernels, thread per row; small ones are CSR (rowOff), whose rows are walked by
  // several lanes each.  nStore is the number of value slots either way.
  std::vector<int> rowOff, sliceOff, col;
  int nStore = 0;
  int maxW = 0;  // SELL: largest slice width
  // restriction to the next level (empty on the coarsest level)
  int nc = 0;
  std::vector<int> agg;            // n: aggregate (coarse row) of each row
  std::vector<int> memOff, mem;    // nc+1 / n: rows of each aggregate
  // gather map producing the next level's values: one list per coarse storage entry
  // (SELL entries, then nc diagonal entries); index >= 0 is a fine off-diagonal storage
  // index, index < 0 encodes fine diagonal row -1-index
  std::vector<int> gOff, gIdx;
};

struct AmgSetupOptions {
  double strength = 0.25;
  int coarseMax = 128;   // dense solve at or below this size
  int maxLevels = 24;
  int passesPerLevel = 2;
  // pairwise passes for the coarsening of level l (l = 0, 1, ...); the last entry repeats, and an
  // empty list means passesPerLevel everywhere
  std::vector<int> passes;
  // coarse levels with more rows than this are stored SELL-32, smaller ones CSR
  int sellMinRows = 65536;
};

// vals / diag are the level-0 matrix in the layout's SELL-32 storage.
std::vector<AmgLevelHost> build_amg_hierarchy(const Layout& L, const std::vector<double>& vals,
                                              const std::vector<double>& diag, const AmgSetupOptions& opt);

}  // namespace anb
