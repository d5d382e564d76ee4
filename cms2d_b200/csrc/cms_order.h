// Host-side construction of the device ordering and the ELL sparsity pattern.
#pragma once
#include <string>
#include <vector>

namespace cms {

// Rows of one group have no couplings among themselves; groups are swept in
// order (forward) and reverse order (backward).  Within a group rows keep the
// natural order.
struct HostPattern {
  int n = 0;          // active cells (unknowns)
  int nD = 0;         // active + dummy cells
  int nmf = 0;        // nmaxfaces
  int G = 0;          // groups (colours or levels)
  int KL = 0, KU = 0; // lower / upper ELL slots (slot s < KL lower, KL <= s < KL+KU upper)
  std::vector<int> gstart;   // [G+1] device-row range of each group
  std::vector<int> gkl, gku; // [G] max lower / upper entries of rows in the group
  std::vector<int> perm;     // [n] device row -> natural cell (0-based)
  std::vector<int> iperm;    // [n] natural cell -> device row
  std::vector<int> col;      // [(KL+KU) * n] device column of slot s of row r (padding: r itself)
  std::vector<signed char> fslot;  // [n * nmf] ELL slot of face k of natural cell i; -1 dummy/none
  std::vector<signed char> nlo, nup;  // [n] lower / upper entry counts per device row
  long long nnz_off = 0;     // stored off-diagonal couplings between active cells
  std::vector<long long> glo, gup;  // [G] lower / upper entries stored in each group
};

// ordering: 0 = greedy multicolour over the natural order, 1 = natural order
// with level scheduling.  cell2cell is 1-based, [nD][nmf] (Fortran (k,i)).
// Returns an empty string on success, else an error message.
std::string build_pattern(int n, int nD, int nmf, const int* cell2cell, const int* ncface, int ordering,
                          HostPattern& out);

}  // namespace cms
