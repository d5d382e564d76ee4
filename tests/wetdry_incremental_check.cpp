// Test program (built and run by tests/test_wetdry.py): the library's
// incremental narrow-channel update (cms::narrow_update) against the full
// recomputation (cms::depth_set + cms::narrow_full) over random batches of
// depth-class changes, including the exact list of cells whose state changed.
// Input: a binary grid dump (n, nD, nmf, ncface, 0-based neighbours,
// directions, depth classes, string cells and dummies); argv[2] = 1 turns the
// narrow-channel switch on.  Prints "bad <count> changes <total>"; exit 0 when
// every batch agrees.
#include <algorithm>
#include <cstdio>
#include <fstream>
#include <random>
#include <vector>

#include "cms_flow_wetdry.h"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  std::ifstream f(argv[1], std::ios::binary);
  int n = 0, nD = 0, nmf = 0;
  f.read((char*)&n, 4); f.read((char*)&nD, 4); f.read((char*)&nmf, 4);
  cms::FlowGeom g;
  g.n = n; g.nD = nD; g.nmf = nmf;
  g.ncface.resize(nD); g.nb.resize((size_t)nD * nmf); g.dir.resize((size_t)nD * nmf);
  std::vector<unsigned char> code(nD);
  f.read((char*)g.ncface.data(), 4 * (size_t)nD);
  f.read((char*)g.nb.data(), 4 * (size_t)nD * nmf);
  f.read((char*)g.dir.data(), 4 * (size_t)nD * nmf);
  f.read((char*)code.data(), nD);
  int nth = 0;
  f.read((char*)&nth, 4);
  cms::WetDryRules R;
  R.closed.assign(nD, 0);
  for (int i = n; i < nD; ++i) R.closed[i] = 1;
  for (int j = 0; j < nth; ++j) {
    int c = 0, d = 0;
    f.read((char*)&c, 4); f.read((char*)&d, 4);
    R.seed_cells.push_back(c); R.seed_dummies.push_back(d); R.closed[d] = 0;
  }
  if (!f) return 2;
  R.narrowchannels = argv[2][0] == '1';
  std::mt19937 rng(7);
  std::vector<unsigned char> w0, pn, w0f, pnf;
  cms::depth_set(g, code.data(), R, w0);
  cms::narrow_full(g, code.data(), R, w0, pn);
  cms::NarrowScratch sc;
  int bad = 0;
  long total = 0;
  for (int it = 0; it < 300; ++it) {
    // scattered changes, or a cluster around one cell (a moving front)
    const int nch = 1 + (int)(rng() % 40), centre = (int)(rng() % nD);
    std::vector<int> ch;
    for (int q = 0; q < nch; ++q) {
      const int x = (it % 3 == 0) ? (int)(rng() % nD) : std::min(nD - 1, std::max(0, centre + (int)(rng() % 200) - 100));
      if (std::find(ch.begin(), ch.end(), x) != ch.end()) continue;
      code[x] = (unsigned char)(rng() % 8);
      ch.push_back(x);
    }
    const std::vector<unsigned char> before = pn;
    std::vector<int> pch;
    cms::narrow_update(g, code.data(), R, ch, w0, pn, sc, pch);
    cms::depth_set(g, code.data(), R, w0f);
    cms::narrow_full(g, code.data(), R, w0f, pnf);
    std::vector<int> real;
    for (int i = 0; i < nD; ++i)
      if (before[i] != pn[i]) real.push_back(i);
    std::sort(pch.begin(), pch.end());
    if (pnf != pn || w0f != w0 || real != pch) ++bad;
    total += (long)real.size();
    for (unsigned char m : sc.mark) if (m) return 3;
    for (unsigned char m : sc.queued) if (m) return 3;
  }
  std::printf("bad %d changes %ld\n", bad, total);
  return bad == 0 ? 0 : 1;
}
