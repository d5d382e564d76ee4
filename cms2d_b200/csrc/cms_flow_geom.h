// Host-side grid metrics of the implicit flow step (natural order, 0-based).
#pragma once
#include <string>
#include <vector>

namespace cms {

// Face arrays are [i * nmf + k] (cell i, face k, both 0-based) over active
// cells; dummies carry no face metrics, as in the reference.
struct FlowGeom {
  int n = 0, nD = 0, nmf = 0;
  std::vector<int> ncface, nb, dir;  // nb: 0-based neighbour (dummies >= n), -1 none; dir 1..4 = N,E,S,W
  std::vector<int> back;             // face index of this face seen from the neighbour (llec2llec - 1)
  std::vector<unsigned char> owned;  // 1: the face is on the cell's no-repeat list (kxyface)
  std::vector<double> x, y, dx, dy, zb, areap;
  std::vector<double> ds, dn, dsxy, fnx, fny, rx, ry, rpx, rpy, dsx, dsy, fintp;
  std::vector<unsigned char> joint;  // joint (refinement-interface) cells
  int njoint = 0;
  double areaavg = 0;
  // cell-based Green-Gauss operator for all cells (ibc = 0): q-th stencil
  // entry of cell i at [i * nsc + q].  The wet-cell operator (ibc = 1) is
  // built and updated on the device from the same metrics.
  int nsc = 0;
  std::vector<int> ga_ncx, ga_ncy, ga_icx, ga_icy;
  std::vector<double> ga_wcx, ga_wcy;
  // cell-reconstruction corrections of joint cells (ider = 2)
  std::vector<int> ga_ngx, ga_ngy, ga_igx, ga_igy;
  std::vector<double> ga_wgxy, ga_wgyx;
  int ider = 1;
  // bit k: face k of the cell takes part in the cell-reconstruction weights
  // (a no-repeat face to an active cell whose size differs by 10 % or more)
  std::vector<unsigned char> crmask;
  std::vector<int> iwet, icorner;
};

// cell2cell/idirface: [nD][nmf] 1-based neighbour ids / direction codes.
// iwet: wet flags of all nD cells.  skewcor: skewness corrections requested.
std::string build_flow_geom(int n, int nD, int nmf, const int* cell2cell, const int* ncface, const int* idirface,
                            const double* x, const double* y, const double* dx, const double* dy, const double* zb,
                            const int* iwet, bool skewcor, FlowGeom& g);

// icorner from g.iwet: wet active cells with more than one dry neighbour
// (flow.F90:1460-1471).
void corner_flags(FlowGeom& g);

}  // namespace cms
