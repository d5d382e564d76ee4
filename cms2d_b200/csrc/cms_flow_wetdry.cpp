// Wetting and drying rules (flow_wetdry(0), source/flow/flow.F90:1231-1539;
// flow_pond, flow.F90:1807-1876) on host arrays in natural order, 0-based.
#include "cms_flow_wetdry.h"

namespace cms {

namespace {

// One visit of the narrow-channel loop (flow.F90:1336-1416, ncellpoly = 0):
// does any removal rule fire for wet cell i?  The two-cell rules count a
// direct neighbour on one side plus the cells beyond the neighbour on the
// other side; the north-north count of the reference is formed but its test
// reads the south count again (flow.F90:1384-1396), so it adds no rule.
bool removal_fires(const FlowGeom& g, const std::vector<int>& w, const unsigned char* code, int i, bool narrow) {
  const int nmf = g.nmf, nf = g.ncface[i];
  const int* nb = &g.nb[(size_t)i * nmf];
  const int* dr = &g.dir[(size_t)i * nmf];
  int ksum = 0;
  for (int k = 0; k < nf; ++k) ksum += w[nb[k]];
  if (narrow) return ksum == 0;  // flow.F90:1325-1341
  if (ksum <= 1) return true;
  int kns = 0, kew = 0;
  for (int k = 0; k < nf; ++k) {
    if (dr[k] == 1 || dr[k] == 3) kns += w[nb[k]];
    if (dr[k] == 2 || dr[k] == 4) kew += w[nb[k]];
  }
  if ((kns == 0 || kew == 0) && (code[i] & WD_LT1)) return true;
  if (!(code[i] & WD_LT2)) return false;
  auto pair_count = [&](int a, int b) {
    int s = 0;
    for (int k = 0; k < nf; ++k) {
      const int c = nb[k];
      if (dr[k] == a) s += w[c];
      if (dr[k] == b)
        for (int kk = 0; kk < g.ncface[c]; ++kk)
          if (g.dir[(size_t)c * nmf + kk] == b) {
            const int c2 = g.nb[(size_t)c * nmf + kk];
            if (c2 >= 0) s += w[c2];
          }
    }
    return s;
  };
  return pair_count(1, 3) == 0 || pair_count(2, 4) == 0 || pair_count(4, 2) == 0;
}

}  // namespace

void wetdry_rules(const FlowGeom& g, const unsigned char* code, const WetDryRules& R, std::vector<int>& iwet) {
  const int n = g.n, nD = g.nD, nmf = g.nmf;
  iwet.assign(nD, 0);
  for (int i = 0; i < nD; ++i) iwet[i] = (code[i] & WD_WET) ? 1 : 0;
  for (int i = 0; i < nD; ++i)
    if (R.closed[i]) iwet[i] = 0;
  // narrow channels: worklist to the fixed point
  std::vector<int> stack;
  std::vector<unsigned char> queued(n, 0);
  stack.reserve(n);
  for (int i = n - 1; i >= 0; --i)
    if (iwet[i]) { stack.push_back(i); queued[i] = 1; }
  auto requeue = [&](int c) {
    if (c >= 0 && c < n && iwet[c] && !queued[c]) { queued[c] = 1; stack.push_back(c); }
  };
  while (!stack.empty()) {
    const int i = stack.back();
    stack.pop_back();
    queued[i] = 0;
    if (!iwet[i] || !removal_fires(g, iwet, code, i, R.narrowchannels)) continue;
    iwet[i] = 0;
    // every cell whose counts include i lies within two faces of it
    for (int k = 0; k < g.ncface[i]; ++k) {
      const int c = g.nb[(size_t)i * nmf + k];
      requeue(c);
      if (c >= 0 && c < n)
        for (int kk = 0; kk < g.ncface[c]; ++kk) requeue(g.nb[(size_t)c * nmf + kk]);
    }
  }
  if (R.ponding) return;
  // flow_pond: wet cells reachable from the string seeds through wet active cells
  std::vector<unsigned char> pond(nD, 0);
  stack.clear();
  for (size_t j = 0; j < R.seed_cells.size(); ++j) {
    const int c = R.seed_cells[j], d = R.seed_dummies[j];
    if (iwet[d]) pond[d] = 1;
    if (iwet[c] && !pond[c]) { pond[c] = 1; stack.push_back(c); }
  }
  while (!stack.empty()) {
    const int i = stack.back();
    stack.pop_back();
    for (int k = 0; k < g.ncface[i]; ++k) {
      const int c = g.nb[(size_t)i * nmf + k];
      if (c < 0 || pond[c] || !iwet[c]) continue;
      pond[c] = 1;
      if (c < n) stack.push_back(c);
    }
  }
  for (int i = 0; i < nD; ++i)
    if (!pond[i]) iwet[i] = 0;
}

}  // namespace cms

#include "cmsgpu.h"

extern "C" int cms_wetdry_rules(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface,
                                const int* idirface, const double* zb, const double* eta, int nth, const int* th_cells,
                                const int* th_faces, double hdry, int ponding, int narrowchannels, int* iwet) {
  if (ncells <= 0 || ncellsD < ncells || nmaxfaces <= 0 || nmaxfaces > 8 || !cell2cell || !ncface || !idirface ||
      !zb || !eta || !iwet || nth < 0 || (nth > 0 && (!th_cells || !th_faces)))
    return CMS_BAD_ARGUMENT;
  cms::FlowGeom g;
  g.n = ncells; g.nD = ncellsD; g.nmf = nmaxfaces;
  g.ncface.assign(ncface, ncface + ncellsD);
  g.nb.resize((size_t)ncellsD * nmaxfaces);
  g.dir.assign(idirface, idirface + (size_t)ncellsD * nmaxfaces);
  for (size_t e = 0; e < g.nb.size(); ++e) {
    g.nb[e] = cell2cell[e] - 1;
    if (g.nb[e] >= ncellsD) return CMS_BAD_ARGUMENT;
  }
  for (int i = 0; i < ncellsD; ++i)
    if (g.ncface[i] < 0 || g.ncface[i] > nmaxfaces) return CMS_BAD_ARGUMENT;
  for (int i = 0; i < ncells; ++i)
    for (int k = 0; k < g.ncface[i]; ++k)
      if (g.nb[(size_t)i * nmaxfaces + k] < 0) return CMS_BAD_ARGUMENT;
  cms::WetDryRules R;
  R.closed.assign(ncellsD, 0);
  for (int i = ncells; i < ncellsD; ++i) R.closed[i] = 1;
  for (int j = 0; j < nth; ++j) {
    const int i = th_cells[j] - 1, k = th_faces[j] - 1;
    if (i < 0 || i >= ncells || k < 0 || k >= nmaxfaces) return CMS_BAD_ARGUMENT;
    const int d = cell2cell[(size_t)i * nmaxfaces + k] - 1;
    if (d < ncells || d >= ncellsD) return CMS_BAD_ARGUMENT;
    R.closed[d] = 0;
    R.seed_cells.push_back(i);
    R.seed_dummies.push_back(d);
  }
  R.ponding = ponding != 0;
  R.narrowchannels = narrowchannels != 0;
  if (hdry <= 0.0) hdry = 0.05;
  const double grav = 9.81, gravinv = 1.0 / 9.81;
  std::vector<unsigned char> code(ncellsD);
  for (int i = 0; i < ncellsD; ++i) {
    const double p = eta[i] * grav;
    const double h = p * gravinv - zb[i];
    code[i] = (unsigned char)((h >= hdry ? cms::WD_WET : 0) | (h < 5.0 * hdry ? cms::WD_LT1 : 0) |
                              (h < 2.0 * hdry ? cms::WD_LT2 : 0));
  }
  std::vector<int> w;
  cms::wetdry_rules(g, code.data(), R, w);
  for (int i = 0; i < ncellsD; ++i) iwet[i] = w[i];
  return CMS_OK;
}
