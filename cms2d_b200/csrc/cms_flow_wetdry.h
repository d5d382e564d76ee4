// Wetting and drying rules of the implicit flow step on host arrays.
#pragma once
#include <vector>

#include "cms_flow_geom.h"

namespace cms {

// Per-cell depth classes from which the rules decide (natural order):
// bit 0 h >= hdry (wet by depth), bit 1 h < hdry1, bit 2 h < hdry2, with
// h = p/g - zb before the hmin floor.
enum { WD_WET = 1, WD_LT1 = 2, WD_LT2 = 4 };

struct WetDryRules {
  std::vector<unsigned char> closed;  // [nD] 1: closed-boundary (wall) dummy, always dry
  std::vector<int> seed_cells, seed_dummies;  // forcing-string cells and their dummies (flow_pond seeds)
  bool ponding = false, narrowchannels = false;
};

// flow_wetdry(0)'s wet set (flow.F90:1231-1539 without structures) from the
// depth classes: depth rule, closed dummies dry, narrow-channel removal
// (Cartesian rules, or the one-cell rule when narrowchannels is on), then
// flow_pond (when ponding is off).  Writes iwet[nD].  The removal rules only
// ever dry cells and each fires on counts of wet cells that can only fall, so
// the reference's repeated sweeps in cell order and the worklist used here end
// at the same set (the largest set on which no rule fires).
void wetdry_rules(const FlowGeom& g, const unsigned char* code, const WetDryRules& R, std::vector<int>& iwet);

}  // namespace cms
