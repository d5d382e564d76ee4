// Grid metrics for the device flow step, computed once per grid on the host.
//
// Restates (0-based, natural order):
//   geo_init_cart       source/geospatial/geospatial.F90:1400-1833 (areas,
//                       back-face links, face lengths, joint cells, no-repeat
//                       face lists, unit normals, distances, skew vectors);
//   interp_coef_cell2face  source/interpolation/interp_lib.f90:2669-2724;
//   der_grad_cbgg       source/derivatives/der_lib.f90:272-378;
//   der_grad_cbggcr     source/derivatives/der_lib.f90:381-443;
//   icorner             source/flow/flow.F90:1460-1471.
#include "cms_flow_geom.h"

#include <algorithm>
#include <cmath>

namespace cms {

namespace {

// keeps stencil entries with |w| > 1e-8 in stencil order (screen_weights,
// der_lib.f90:681-715); returns the count
int keep_nonzero(int nt, const double* w, const int* idx, int* out_i, double* out_w) {
  int c = 0;
  for (int k = 0; k <= nt; ++k)
    if (std::fabs(w[k]) > 1.0e-8) { out_i[c] = idx[k]; out_w[c] = w[k]; ++c; }
  return c;
}

}  // namespace

std::string build_flow_geom(int n, int nD, int nmf, const int* cell2cell, const int* ncface, const int* idirface,
                            const double* x, const double* y, const double* dx, const double* dy, const double* zb,
                            const int* iwet, bool skewcor, FlowGeom& g) {
  if (n <= 0 || nD < n || nmf <= 0 || nmf > 8) return "bad grid sizes";
  g.n = n; g.nD = nD; g.nmf = nmf;
  const size_t NFc = (size_t)nD * nmf;
  g.ncface.assign(ncface, ncface + nD);
  g.x.assign(x, x + nD); g.y.assign(y, y + nD); g.dx.assign(dx, dx + nD); g.dy.assign(dy, dy + nD);
  g.zb.assign(zb, zb + nD);
  g.iwet.assign(iwet, iwet + nD);
  g.nb.assign(NFc, -1); g.dir.assign(NFc, 0); g.back.assign(NFc, -1); g.owned.assign(NFc, 0);
  for (auto* v : {&g.ds, &g.dn, &g.dsxy, &g.fnx, &g.fny, &g.rx, &g.ry, &g.rpx, &g.rpy, &g.dsx, &g.dsy, &g.fintp})
    v->assign(NFc, 0.0);
  g.areap.resize(nD);
  for (int i = 0; i < nD; ++i) g.areap[i] = dx[i] * dy[i];
  double asum = 0;
  for (int i = 0; i < n; ++i) asum += g.areap[i];
  g.areaavg = asum / (double)n;
  auto at = [nmf](int i, int k) { return (size_t)i * nmf + k; };
  for (int i = 0; i < nD; ++i) {
    for (int k = 0; k < nmf; ++k) {
      g.nb[at(i, k)] = cell2cell[at(i, k)] - 1;
      g.dir[at(i, k)] = idirface[at(i, k)];
    }
  }
  static const int opposite[5] = {0, 3, 4, 1, 2};
  // back links and face lengths (active cells)
  for (int i = 0; i < n; ++i) {
    if (g.ncface[i] < 1 || g.ncface[i] > nmf) return "ncface out of range";
    for (int k = 0; k < g.ncface[i]; ++k) {
      const int j = g.nb[at(i, k)], d = g.dir[at(i, k)];
      if (j < 0 || j >= nD || d < 1 || d > 4) return "bad connectivity or face direction";
      if (j < n) {
        for (int kk = 0; kk < g.ncface[j]; ++kk)
          if (g.nb[at(j, kk)] == i) g.back[at(i, k)] = kk;
      } else {
        g.back[at(i, k)] = opposite[d] - 1;
      }
      if (g.back[at(i, k)] < 0) return "neighbour does not link back";
      g.ds[at(i, k)] = (d == 1 || d == 3) ? std::min(dx[i], dx[j]) : std::min(dy[i], dy[j]);
    }
  }
  // joint cells: a same-direction neighbour of a different size (ratio outside [0.8, 1.2])
  g.joint.assign(nD, 0);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < g.ncface[i]; ++k) {
      const int j = g.nb[at(i, k)], d = g.dir[at(i, k)];
      if (j >= n) continue;
      const double r = (d == 2 || d == 4) ? dy[i] / dy[j] : dx[i] / dx[j];
      if (r > 1.2 || r < 0.8) g.joint[i] = g.joint[j] = 1;
    }
  g.njoint = 0;
  for (int i = 0; i < n; ++i) g.njoint += g.joint[i];
  // no-repeat faces: a face belongs to the first cell (in natural order) that visits it
  {
    std::vector<unsigned char> seen(NFc, 0);
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < g.ncface[i]; ++k) {
        if (seen[at(i, k)]) continue;
        seen[at(i, k)] = 1;
        seen[at(g.nb[at(i, k)], g.back[at(i, k)])] = 1;
        g.owned[at(i, k)] = 1;
      }
  }
  // normals, normal distances, centre-to-face vectors, skew parts
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < g.ncface[i]; ++k) {
      const size_t f = at(i, k);
      const int j = g.nb[f], d = g.dir[f];
      const double nx = d == 2 ? 1.0 : d == 4 ? -1.0 : 0.0;
      const double ny = d == 1 ? 1.0 : d == 3 ? -1.0 : 0.0;
      g.fnx[f] = nx; g.fny[f] = ny;
      if (d == 1 || d == 3) {
        g.dn[f] = std::fabs(y[j] - y[i]);
        g.rx[f] = x[j] - x[i];
        g.ry[f] = (d == 1 ? 1.0 : -1.0) * dy[i] / 2.0;
      } else {
        g.dn[f] = std::fabs(x[j] - x[i]);
        g.rx[f] = (d == 2 ? 1.0 : -1.0) * dx[i] / 2.0;
        g.ry[f] = y[j] - y[i];
      }
      g.rpx[f] = g.rx[f] - nx * std::fabs(g.rx[f]);
      g.rpy[f] = g.ry[f] - ny * std::fabs(g.ry[f]);
      g.dsx[f] = nx * g.ds[f];
      g.dsy[f] = ny * g.ds[f];
      g.dsxy[f] = g.ds[f] / g.dn[f];
      // interpolation weight of the neighbour
      if (!g.joint[i]) {
        const int jj = g.nb[at(i, k)];
        g.fintp[f] = (k == 0 || k == 2) ? dy[i] / (dy[i] + dy[jj]) : dx[i] / (dx[i] + dx[jj]);
      } else {
        g.fintp[f] = (d == 2 || d == 4) ? dx[i] / (dx[i] + dx[j]) : dy[i] / (dy[i] + dy[j]);
      }
    }
  // Green-Gauss operator of all cells (the wet-cell one is built on the device)
  g.nsc = nmf + 1;
  g.ider = (skewcor && g.njoint > 0) ? 2 : 1;
  const int nsc = g.nsc;
  auto gg = [&](int ibc, std::vector<int>& ncx, std::vector<int>& ncy, std::vector<int>& icx, std::vector<int>& icy,
                std::vector<double>& wcx, std::vector<double>& wcy, std::vector<int>& ngx, std::vector<int>& ngy,
                std::vector<int>& igx, std::vector<int>& igy, std::vector<double>& wgxy, std::vector<double>& wgyx) {
    ncx.assign(n, 0); ncy.assign(n, 0);
    icx.assign((size_t)n * nsc, 0); icy = icx;
    wcx.assign((size_t)n * nsc, 0.0); wcy = wcx;
    ngx.assign(n, 0); ngy.assign(n, 0);
    igx.assign((size_t)n * nsc, 0); igy = igx;
    wgxy.assign((size_t)n * nsc, 0.0); wgyx = wgxy;
    std::vector<double> tx(nmf + 1), ty(nmf + 1);
    std::vector<int> ti(nmf + 1), tj(nmf + 1);
    for (int i = 0; i < n; ++i) {
      if (g.iwet[i] == 0 && ibc == 1) continue;
      std::fill(tx.begin(), tx.end(), 0.0);
      std::fill(ty.begin(), ty.end(), 0.0);
      ti[0] = i; tj[0] = i;
      for (int k = 0; k < g.ncface[i]; ++k) {
        const size_t f = at(i, k);
        const int j = g.nb[f];
        ti[k + 1] = j; tj[k + 1] = j;
        if (g.iwet[j] == 1 || ibc == 0) {
          tx[0] += g.dsx[f] * (1.0 - g.fintp[f]);
          tx[k + 1] = g.dsx[f] * g.fintp[f];
          ty[0] += g.dsy[f] * (1.0 - g.fintp[f]);
          ty[k + 1] = g.dsy[f] * g.fintp[f];
        } else {
          tx[0] += g.dsx[f];
          ty[0] += g.dsy[f];
        }
      }
      for (int k = 0; k <= nmf; ++k) { tx[k] /= g.areap[i]; ty[k] /= g.areap[i]; }
      ncx[i] = keep_nonzero(nmf, tx.data(), ti.data(), &icx[(size_t)i * nsc], &wcx[(size_t)i * nsc]);
      ncy[i] = keep_nonzero(nmf, ty.data(), tj.data(), &icy[(size_t)i * nsc], &wcy[(size_t)i * nsc]);
      // remove the mean so that each stencil sums to zero
      double sx = 0, sy = 0;
      for (int q = 0; q < ncx[i]; ++q) sx += wcx[(size_t)i * nsc + q];
      for (int q = 0; q < ncy[i]; ++q) sy += wcy[(size_t)i * nsc + q];
      for (int q = 0; q < ncx[i]; ++q) wcx[(size_t)i * nsc + q] -= sx / (double)ncx[i];
      for (int q = 0; q < ncy[i]; ++q) wcy[(size_t)i * nsc + q] -= sy / (double)ncy[i];
    }
    if (g.ider != 2) return;
    for (int i = 0; i < n; ++i) {
      if (!g.joint[i]) continue;
      if (g.iwet[i] == 0 && ibc == 1) continue;
      std::fill(tx.begin(), tx.end(), 0.0);
      std::fill(ty.begin(), ty.end(), 0.0);
      ti.assign(nmf + 1, 0); tj.assign(nmf + 1, 0);
      ti[0] = i; tj[0] = i;
      for (int k = 0; k < g.ncface[i]; ++k) {
        const size_t f = at(i, k);
        if (!g.owned[f]) continue;
        const int j = g.nb[f], d = g.dir[f];
        const bool xface = (d == 2 || d == 4);
        if (!xface) tj[k + 1] = j;
        const double ratio = xface ? dy[i] / dy[std::min(j, nD - 1)] : dx[i] / dx[std::min(j, nD - 1)];
        if (j >= n || std::fabs(ratio - 1.0) < 0.1) continue;
        if (g.iwet[j] == 0 && ibc == 1) continue;
        const size_t fb = at(j, g.back[f]);
        if (xface) {
          tx[0] += g.dsx[f] * (1.0 - g.fintp[f]) * g.rpy[f] / g.areap[i];
          tx[k + 1] = g.dsx[f] * g.fintp[f] * g.rpy[fb] / g.areap[i];
          ti[k + 1] = j;
        } else {
          ty[0] += g.dsy[f] * (1.0 - g.fintp[f]) * g.rpx[f] / g.areap[i];
          ty[k + 1] = g.dsy[f] * g.fintp[f] * g.rpx[fb] / g.areap[i];
        }
      }
      ngx[i] = keep_nonzero(nmf, tx.data(), ti.data(), &igx[(size_t)i * nsc], &wgxy[(size_t)i * nsc]);
      ngy[i] = keep_nonzero(nmf, ty.data(), tj.data(), &igy[(size_t)i * nsc], &wgyx[(size_t)i * nsc]);
    }
  };
  gg(0, g.ga_ncx, g.ga_ncy, g.ga_icx, g.ga_icy, g.ga_wcx, g.ga_wcy, g.ga_ngx, g.ga_ngy, g.ga_igx, g.ga_igy, g.ga_wgxy,
     g.ga_wgyx);
  // faces of the cell-reconstruction weights (der_grad_cbggcr's skip test)
  g.crmask.assign(nD, 0);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < g.ncface[i]; ++k) {
      const size_t f = at(i, k);
      if (!g.owned[f]) continue;
      const int j = g.nb[f], d = g.dir[f];
      if (j >= n) continue;
      const double ratio = (d == 2 || d == 4) ? dy[i] / dy[j] : dx[i] / dx[j];
      if (std::fabs(ratio - 1.0) < 0.1) continue;
      g.crmask[i] |= (unsigned char)(1u << k);
    }
  corner_flags(g);
  return std::string();
}

void corner_flags(FlowGeom& g) {
  const int n = g.n, nmf = g.nmf;
  g.icorner.assign(g.nD, 0);
  for (int i = 0; i < n; ++i) {
    if (g.iwet[i] != 1) continue;
    int nd = 0;
    for (int k = 0; k < g.ncface[i]; ++k) nd += (g.iwet[g.nb[(size_t)i * nmf + k]] == 0);
    g.icorner[i] = nd > 1;
  }
}

}  // namespace cms
