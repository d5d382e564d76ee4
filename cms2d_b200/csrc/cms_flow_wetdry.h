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

// flow_wetdry(0)'s wet set in three stages (flow.F90:1231-1539 without
// structures), all arrays natural order over nD cells:
//   depth_set    the depth rule with closed dummies dry (w0);
//   narrow_full  the narrow-channel removal (Cartesian rules, or the one-cell
//                rule with narrowchannels) from w0 (pn);
//   pond_host    flow_pond: cells of pn not reachable from the string seeds
//                through wet active cells are dried (iwet; skipped with ponding).
// The removal rules only ever dry cells and each fires on counts of wet cells
// that can only fall, so the reference's repeated sweeps in cell order and
// the worklist used here end at the same set (the largest set on which no
// rule fires).
void depth_set(const FlowGeom& g, const unsigned char* code, const WetDryRules& R, std::vector<unsigned char>& w0);
void narrow_full(const FlowGeom& g, const unsigned char* code, const WetDryRules& R,
                 const std::vector<unsigned char>& w0, std::vector<unsigned char>& pn);
void pond_host(const FlowGeom& g, const WetDryRules& R, const std::vector<unsigned char>& pn, std::vector<int>& iwet);
// All three stages.
void wetdry_rules(const FlowGeom& g, const unsigned char* code, const WetDryRules& R, std::vector<int>& iwet);

// Incremental narrow-channel update after the depth classes of the cells in
// `changed` (natural ids, codes already updated) changed: w0 and pn are
// brought to what depth_set and narrow_full would give for the new classes,
// and the cells whose pn changed are appended to pchanged.  Work is
// proportional to the changed cells and the removed regions around them:
// a previously removed cell can only come back if a chain of removed cells,
// each within two faces of the next, links it to a cell whose class changed
// (otherwise the removals that justified it still hold), and a kept cell can
// only start to fire if its class changed or a cell within two faces left.
struct NarrowScratch {
  std::vector<unsigned char> mark, queued;  // [nD] zeroed between calls
  std::vector<int> list, stack;
};
void narrow_update(const FlowGeom& g, const unsigned char* code, const WetDryRules& R,
                   const std::vector<int>& changed, std::vector<unsigned char>& w0, std::vector<unsigned char>& pn,
                   NarrowScratch& sc, std::vector<int>& pchanged);

}  // namespace cms
