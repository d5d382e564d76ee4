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
template <typename W>
bool removal_fires(const FlowGeom& g, const W& w, const unsigned char* code, int i, bool narrow) {
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

// calls f(c) for the active cells within two faces of active cell i (i included)
template <typename Fn>
void within_two(const FlowGeom& g, int i, Fn f) {
  const int n = g.n, nmf = g.nmf;
  f(i);
  for (int k = 0; k < g.ncface[i]; ++k) {
    const int c = g.nb[(size_t)i * nmf + k];
    if (c < 0 || c >= n) continue;
    f(c);
    for (int kk = 0; kk < g.ncface[c]; ++kk) {
      const int c2 = g.nb[(size_t)c * nmf + kk];
      if (c2 >= 0 && c2 < n) f(c2);
    }
  }
}

// removals to the fixed point from the queued cells (worklist)
void remove_to_fixed_point(const FlowGeom& g, const unsigned char* code, bool narrow, std::vector<unsigned char>& pn,
                           std::vector<int>& stack, std::vector<unsigned char>& queued, std::vector<int>* removed) {
  while (!stack.empty()) {
    const int i = stack.back();
    stack.pop_back();
    queued[i] = 0;
    if (!pn[i] || !removal_fires(g, pn, code, i, narrow)) continue;
    pn[i] = 0;
    if (removed) removed->push_back(i);
    // every cell whose counts include i lies within two faces of it
    within_two(g, i, [&](int c) {
      if (pn[c] && !queued[c]) { queued[c] = 1; stack.push_back(c); }
    });
  }
}

}  // namespace

void depth_set(const FlowGeom& g, const unsigned char* code, const WetDryRules& R, std::vector<unsigned char>& w0) {
  w0.assign(g.nD, 0);
  for (int i = 0; i < g.nD; ++i) w0[i] = (!R.closed[i] && (code[i] & WD_WET)) ? 1 : 0;
}

void narrow_full(const FlowGeom& g, const unsigned char* code, const WetDryRules& R,
                 const std::vector<unsigned char>& w0, std::vector<unsigned char>& pn) {
  const int n = g.n;
  pn = w0;
  std::vector<int> stack;
  std::vector<unsigned char> queued(g.nD, 0);
  stack.reserve(n);
  for (int i = n - 1; i >= 0; --i)
    if (pn[i]) { stack.push_back(i); queued[i] = 1; }
  remove_to_fixed_point(g, code, R.narrowchannels, pn, stack, queued, nullptr);
}

void pond_host(const FlowGeom& g, const WetDryRules& R, const std::vector<unsigned char>& pn, std::vector<int>& iwet) {
  const int n = g.n, nD = g.nD, nmf = g.nmf;
  iwet.assign(nD, 0);
  for (int i = 0; i < nD; ++i) iwet[i] = pn[i];
  if (R.ponding) return;
  // flow_pond: wet cells reachable from the string seeds through wet active cells
  std::vector<unsigned char> pond(nD, 0);
  std::vector<int> stack;
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

void wetdry_rules(const FlowGeom& g, const unsigned char* code, const WetDryRules& R, std::vector<int>& iwet) {
  std::vector<unsigned char> w0, pn;
  depth_set(g, code, R, w0);
  narrow_full(g, code, R, w0, pn);
  pond_host(g, R, pn, iwet);
}

void narrow_update(const FlowGeom& g, const unsigned char* code, const WetDryRules& R,
                   const std::vector<int>& changed, std::vector<unsigned char>& w0, std::vector<unsigned char>& pn,
                   NarrowScratch& sc, std::vector<int>& pchanged) {
  const int n = g.n, nD = g.nD;
  if ((int)sc.mark.size() != nD) { sc.mark.assign(nD, 0); sc.queued.assign(nD, 0); }
  std::vector<int>& cand = sc.list;
  std::vector<int>& stack = sc.stack;
  cand.clear();
  stack.clear();
  // new depth set; dummies take it as their final state (no rule touches
  // them), and a dummy that changes acts on the cells within two faces of it
  // through its cell
  std::vector<int> leavers, wetter_dummies;
  for (int x : changed) {
    const unsigned char nw = (!R.closed[x] && (code[x] & WD_WET)) ? 1 : 0;
    w0[x] = nw;
    if (x >= n) {
      if (pn[x] != nw) {
        pn[x] = nw;
        pchanged.push_back(x);
        (nw ? wetter_dummies : leavers).push_back(x);
      }
      continue;
    }
    if (pn[x] && !nw) leavers.push_back(x);
  }
  auto around = [&](int x, auto f) {  // cells within two faces of x (through its cell for a dummy)
    if (x < n) { within_two(g, x, f); return; }
    for (int k = 0; k < g.ncface[x]; ++k) {
      const int c = g.nb[(size_t)x * g.nmf + k];
      if (c >= 0 && c < n) within_two(g, c, f);
    }
  };
  // candidates: removed (or newly depth-wet) cells linked to a changed cell
  // through removed cells within two faces of each other
  auto removed_cell = [&](int c) { return w0[c] && !pn[c]; };
  for (int x : changed)
    if (x < n && removed_cell(x) && !sc.mark[x]) { sc.mark[x] = 1; cand.push_back(x); }
  for (int x : wetter_dummies)
    around(x, [&](int c) {
      if (!sc.mark[c] && removed_cell(c)) { sc.mark[c] = 1; cand.push_back(c); }
    });
  for (size_t q = 0; q < cand.size(); ++q)
    within_two(g, cand[q], [&](int c) {
      if (!sc.mark[c] && removed_cell(c)) { sc.mark[c] = 1; cand.push_back(c); }
    });
  // tentative set: previous kept cells minus leavers plus candidates
  for (int x : leavers)
    if (x < n) { pn[x] = 0; pchanged.push_back(x); }
  for (int c : cand) {
    sc.mark[c] = 0;
    pn[c] = 1;
    if (!sc.queued[c]) { sc.queued[c] = 1; stack.push_back(c); }
  }
  auto enqueue = [&](int c) {
    if (pn[c] && !sc.queued[c]) { sc.queued[c] = 1; stack.push_back(c); }
  };
  for (int x : changed)
    if (x < n) enqueue(x);
  for (int x : leavers) around(x, enqueue);
  std::vector<int> removed;
  remove_to_fixed_point(g, code, R.narrowchannels, pn, stack, sc.queued, &removed);
  // net changes of the candidates: re-added ones that stayed, and removals of
  // cells that were kept before (a candidate removed again is no change)
  for (int c : cand) sc.mark[c] = 1;
  for (int c : cand)
    if (pn[c]) pchanged.push_back(c);
  for (int x : removed)
    if (!sc.mark[x]) pchanged.push_back(x);
  for (int c : cand) sc.mark[c] = 0;
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
