// Device ordering and ELL pattern for the ILU(0)-preconditioned Krylov solves.
//
// The reference factorises and sweeps in the natural cell order
// (source/solvers/ilu0.f90:2-65, sparse.f90:237-264), a strict row-by-row
// recurrence.  On the GPU the unknowns are renumbered so that each sweep
// becomes a short sequence of fully parallel groups:
//   * multicolour: greedy colouring in natural order (two colours -- red/black
//     -- on a Cartesian 5-point grid, a few more at telescoping interfaces);
//     ILU(0) of the permuted matrix P A P^T, a different preconditioner whose
//     iteration counts are reported against the natural order;
//   * natural: level scheduling of the natural-order lower-triangular
//     dependency graph; rows are regrouped by level, which leaves every row's
//     lower/upper neighbour sets unchanged, so the factor and the sweeps are
//     the natural-order ILU(0) up to the order of floating-point additions.
// The pattern keeps only couplings between active cells, as indexm does
// (sparse.f90:45); dummy-cell terms enter the right-hand side instead.
#include "cms_order.h"

#include <algorithm>
#include <cstdio>

namespace cms {

std::string build_pattern(int n, int nD, int nmf, const int* cell2cell, const int* ncface, int ordering,
                          HostPattern& P) {
  if (n <= 0 || nD < n || nmf <= 0 || nmf > 8) return "bad grid sizes";
  P.n = n; P.nD = nD; P.nmf = nmf;
  // interior adjacency (0-based), in face order
  std::vector<int> adj((size_t)n * nmf, -1);
  for (int i = 0; i < n; ++i) {
    int nf = ncface[i];
    if (nf < 0 || nf > nmf) return "ncface out of range";
    for (int k = 0; k < nf; ++k) {
      int c = cell2cell[(size_t)i * nmf + k];
      if (c < 1 || c > nD) return "cell2cell of an active cell out of range";
      if (c <= n) {
        if (c - 1 == i) return "a cell is its own neighbour";
        for (int kk = 0; kk < k; ++kk)
          if (adj[(size_t)i * nmf + kk] == c - 1) return "repeated neighbour in cell2cell";
        adj[(size_t)i * nmf + k] = c - 1;
      }
    }
  }
  // groups
  std::vector<int> grp(n, 0);
  if (ordering == 0) {
    std::vector<int> mark(64, -1);
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < nmf; ++k) {
        int j = adj[(size_t)i * nmf + k];
        if (j >= 0 && j < i) mark[grp[j]] = i;
      }
      int c = 0;
      while (mark[c] == i) ++c;
      if (c >= 63) return "colouring needs too many colours";
      grp[i] = c;
    }
  } else {
    for (int i = 0; i < n; ++i) {
      int l = 0;
      for (int k = 0; k < nmf; ++k) {
        int j = adj[(size_t)i * nmf + k];
        if (j >= 0 && j < i) l = std::max(l, grp[j] + 1);
      }
      grp[i] = l;
    }
  }
  int G = 0;
  for (int i = 0; i < n; ++i) G = std::max(G, grp[i] + 1);
  P.G = G;
  // counting sort by group (stable: natural order inside a group)
  P.gstart.assign(G + 1, 0);
  for (int i = 0; i < n; ++i) P.gstart[grp[i] + 1]++;
  for (int g = 0; g < G; ++g) P.gstart[g + 1] += P.gstart[g];
  P.perm.assign(n, 0);
  P.iperm.assign(n, 0);
  {
    std::vector<int> pos(P.gstart.begin(), P.gstart.end() - 1);
    for (int i = 0; i < n; ++i) {
      int r = pos[grp[i]]++;
      P.perm[r] = i;
      P.iperm[i] = r;
    }
  }
  // lower / upper entries per device row, ascending device column
  std::vector<int> lo((size_t)n * nmf), up((size_t)n * nmf);
  std::vector<int> lofc((size_t)n * nmf), upfc((size_t)n * nmf);  // face of each entry
  P.nlo.assign(n, 0);
  P.nup.assign(n, 0);
  P.gkl.assign(G, 0);
  P.gku.assign(G, 0);
  P.glo.assign(G, 0);
  P.gup.assign(G, 0);
  int KL = 0, KU = 0;
  long long nnz = 0;
  for (int r = 0; r < n; ++r) {
    int i = P.perm[r];
    int nl = 0, nu = 0;
    std::pair<int, int> L[8], U[8];
    for (int k = 0; k < nmf; ++k) {
      int j = adj[(size_t)i * nmf + k];
      if (j < 0) continue;
      int cj = P.iperm[j];
      if (cj < r) L[nl++] = {cj, k}; else U[nu++] = {cj, k};
    }
    std::sort(L, L + nl);
    std::sort(U, U + nu);
    for (int t = 0; t < nl; ++t) { lo[(size_t)r * nmf + t] = L[t].first; lofc[(size_t)r * nmf + t] = L[t].second; }
    for (int t = 0; t < nu; ++t) { up[(size_t)r * nmf + t] = U[t].first; upfc[(size_t)r * nmf + t] = U[t].second; }
    P.nlo[r] = (signed char)nl;
    P.nup[r] = (signed char)nu;
    int g = grp[i];
    P.glo[g] += nl;
    P.gup[g] += nu;
    P.gkl[g] = std::max(P.gkl[g], nl);
    P.gku[g] = std::max(P.gku[g], nu);
    KL = std::max(KL, nl);
    KU = std::max(KU, nu);
    nnz += nl + nu;
  }
  P.KL = KL; P.KU = KU; P.nnz_off = nnz;
  const int K = KL + KU;
  P.col.assign((size_t)std::max(K, 1) * n, 0);
  P.fslot.assign((size_t)n * nmf, (signed char)-1);
  for (int r = 0; r < n; ++r) {
    int i = P.perm[r];
    for (int s = 0; s < K; ++s) P.col[(size_t)s * n + r] = r;  // padding: the row itself, value 0
    for (int t = 0; t < P.nlo[r]; ++t) {
      P.col[(size_t)t * n + r] = lo[(size_t)r * nmf + t];
      P.fslot[(size_t)i * nmf + lofc[(size_t)r * nmf + t]] = (signed char)t;
    }
    for (int t = 0; t < P.nup[r]; ++t) {
      P.col[(size_t)(KL + t) * n + r] = up[(size_t)r * nmf + t];
      P.fslot[(size_t)i * nmf + upfc[(size_t)r * nmf + t]] = (signed char)(KL + t);
    }
  }
  return std::string();
}

}  // namespace cms
