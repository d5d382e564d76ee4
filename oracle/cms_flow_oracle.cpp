// CPU oracle of one CMS-Flow implicit time step (test infrastructure only).
//
// Plain C++ restatement of flow_imp (source/flow/flow_imp.F90:29-312) and the
// routines it calls for the configurations this build covers: Cartesian and
// telescoping grids (simple and joint cells, skewness corrections), ntsch = 1,
// exponential convection scheme (ndsch = 4), Manning friction without waves,
// the mturbul = 5 eddy viscosity, tidal/water-level (TH/H) boundary strings and
// walls, wetting and drying (flow_wetdry(0) with flow_pond, der_update).
// Water levels on boundary strings are inputs of a step (bnd_eval stays with
// the caller).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline load it.
// Arrays are 1-based like the Fortran: index 0 is unused; face arrays are
// [(i)*NF + k] with NF = nmaxfaces + 1.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

extern "C" {
void* orc_create(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface, const int* iwet,
                 int fix_last_cell);
void orc_destroy(void* h);
void orc_set_wet(void* h, const int* iwet);
int orc_solve_d(void* hv, const double* acoef, double* ss, const double* sp, double* res, double* phi, double relax,
                int nswp, int nsolv, int precond, double tol, int lfil, double droptol, double permtol, double* rmom,
                int* iters, int* inner, double* relres, int norm);
int orc_solve_n_d(void* hv, int n, const double* acoef, double* ss, const double* sp, double* res, double* phi,
                  double relax, int nswp, int nsolv, double relaxsor, int nswp0_vel, int precond, double tol,
                  double* rmom, int* iters, int* inner, double* relres, int norm);
}

namespace {

using V = std::vector<double>;
using VI = std::vector<int>;

struct Params {
  double grav = 9.81;             // flow.F90:34
  double hmin = 0.05, hdry = 0.05;  // flow.F90:50-51
  double hdry1 = 0.25, hdry2 = 0.1;  // 5 hdry, 2 hdry (flow.F90:52-53, 686-689)
  double small = 1.0e-15;          // definitions.F90:93
  bool ponding = false, narrowchannels = false;  // flow.F90:54-55
  double relax_uv = 0.8, relax_pp = 1.0, relax_p = 1.0;  // flow.F90:124-130
  double facpp = 0.2;             // flow.F90:132
  double cviscon = 1.0e-6, cvisbot = 0.0667, cvishor = 0.2, cvismax = 20.0;  // flow.F90:82-96 (mturbul=5)
  double wallfac = 1.0;           // friction.F90:49
  double rmommaxp = 1e-3, rmomtargetp = 1e-4, rmomminp = 1e-8, rmomratiop = 0.5;      // flow.F90:135-150
  double rmommaxuv = 1e-2, rmomtargetuv = 1e-3, rmomminuv = 1e-7, rmomratiouv = 1.0;
  int dtvar = 0;                  // fixed time step in this build
  int ndsch = 4;                  // advection scheme, exponential (flow.F90:111)
};

struct Flow {
  int n = 0, nD = 0, nmf = 0, NF = 0;
  bool skewcor = true;
  Params P;
  // grid
  VI c2c, ncface, idir;  // face arrays [(i)*NF+k]
  V x, y, dx, dy, zb;
  // geometry
  V areap, ds, dn, dsxy, fnx, fny, rx, ry, rpx, rpy, dsx, dsy, fintp, zbk;
  VI llec, nxyface, kxyface, nxface, kxface, nyface, kyface;
  VI isjoint, idjoint;
  double areaavg = 0, cvishor2areaavg = 0;
  // gradient operators: gow (ibc=1, wet cells), goa (ibc=0)
  struct GO {
    int nsc = 0;
    VI ncx, ncy, icx, icy;  // [(i)*nsc + q], q = 1..nsc
    V wcx, wcy;
    VI ngx, ngy, igx, igy;
    V wgxy, wgyx;
    int ider = 1;
  } gow, goa;
  // state
  VI iwet, iwet1, icorner;
  int last_nlist = 0;  // cells der_update recomputed in the last step
  V p, h, u, v, pp, eta, vis, cfrict, uelwc, uv, bsxy, bsvel, z0, coefman, cmb, fc;
  V u1, v1, p1, h1;
  V flux, visk, hk, pk, acoef;
  V su, sv, sp, spu, spv, ssu0, ssv0, spuv0, sppp0, sspp0, apuareap, sumu, Hu, Hv, cbcfuwcap;
  V dpx, dpy, dux, duy, dvx, dvy, dppx, dppy, dHux, dHuy, dHvx, dHvy, dapx, dapy, dzbx, dzby;
  V rsu, rsv, rsp;
  double rmom[4] = {0, 0, 0, 0}, rmom0[4] = {0, 0, 0, 0}, rmom1[4] = {0, 0, 0, 0};
  // boundary strings
  VI th_cells, th_faces;  // TH/H water-level string (1-based cells, faces)
  VI w_cells, w_faces;    // wall string
  V wsebnd;
  void* solver = nullptr;
  // optional unknown ordering of the solves: row r of the solver is natural
  // cell perm[r] (0-based); dummies keep their numbers
  std::vector<int> perm, iperm;
  void* solver_perm = nullptr;
  // solver settings
  int nsolv = 4, precond = 1, nswp_pp = 20, nswp_uv = 5, norm = 1;
  double relaxsor = 1.8;  // SOR constant of nsolv 2 and 5 (flow.F90:131)
  double tol = 1e-3;
  int last_niter = 0, last_iconv = 1;
  long long solve_iters = 0;
  // capture of one assembled system (the iteration-count report): the next
  // solve of variable cap_var is copied, natural order, before it runs
  int cap_var = 0, cap_done = 0;
  V cap_acoef, cap_ss, cap_sp, cap_phi;

  inline int& C(int k, int i) { return c2c[(size_t)i * NF + k]; }
  inline double& F(V& a, int k, int i) { return a[(size_t)i * NF + k]; }
  inline int& FI(VI& a, int k, int i) { return a[(size_t)i * NF + k]; }
};

double exponentialcoef(double dk, double fk) {  // comp_lib.f90:96-109
  double absfk = std::fabs(fk);
  double peck = absfk / std::max(std::max(dk, 1.0e-6), absfk);
  return dk * peck / std::max(std::exp(peck) - 1.0, 1.0e-6) + std::max(0.0, -fk);
}
double upwindcoef(double dk, double fk) { return dk + std::max(0.0, -fk); }  // comp_lib.f90:54-64
double hybridcoef(double dk, double fk) {  // comp_lib.f90:67-78
  double peck = std::fabs(fk) / std::max(dk, 1.0e-6);
  return dk * std::max(0.0, 1.0 - 0.5 * peck) + std::max(0.0, -fk);
}
double powerlawcoef(double dk, double fk) {  // comp_lib.f90:81-93
  double absfk = std::fabs(fk);
  double peck = absfk / std::max(std::max(dk, absfk), 1.0e-6);
  double p2 = peck * peck;
  return dk * (1.0 - p2 * p2 * peck) + std::max(0.0, -fk);
}
// the coefficient function flow_imp passes to coeffsourcesink_uv (flow_imp.F90:120-126)
double schemecoef(int ndsch, double dk, double fk) {
  switch (ndsch) {
    case 0: return 0.0;  // zerocoef (comp_lib.f90:40-51)
    case 2: return hybridcoef(dk, fk);
    case 3: return powerlawcoef(dk, fk);
    case 4: return exponentialcoef(dk, fk);
    default: return upwindcoef(dk, fk);
  }
}
double wall_coef(double yp, double y0) {  // fric_lib.f90:162-194
  double y0lim = std::min(std::max(y0, 1.0e-6), yp * 0.9999);
  double c = 0.4 / std::log(yp / y0lim);
  return c * c;
}
double man2drag(double g, double cman, double h, double hmax) {  // fric_lib.f90:944-969
  double hh = std::max(std::min(hmax, h), 0.1 * cman);
  return g * cman * cman / std::pow(hh, 0.3333);
}
double drag2length(double Cd, double h) {  // fric_lib.f90:972-996
  double z0 = h / std::exp(0.4 / std::sqrt(Cd) + 1.0);
  return std::max(z0, 1.0e-6);
}

// geo_init_cart (geospatial.F90:1400-1833) and interp_coef_cell2face
// (interp_lib.f90:2669-2724): metrics of active cells' faces.
void geometry(Flow& f) {
  const int n = f.n, nD = f.nD, NF = f.NF;
  f.areap.assign(nD + 1, 0.0);
  for (int i = 1; i <= nD; ++i) f.areap[i] = f.dx[i] * f.dy[i];
  double s = 0;
  for (int i = 1; i <= n; ++i) s += f.areap[i];
  f.areaavg = s / (double)n;
  f.cvishor2areaavg = f.P.cvishor * f.P.cvishor * f.areaavg;  // flow.F90:739
  size_t FS = (size_t)(nD + 1) * NF;
  for (V* a : {&f.ds, &f.dn, &f.dsxy, &f.fnx, &f.fny, &f.rx, &f.ry, &f.rpx, &f.rpy, &f.dsx, &f.dsy, &f.fintp})
    a->assign(FS, 0.0);
  f.llec.assign(FS, 0);
  for (int i = 1; i <= n; ++i) {
    for (int k = 1; k <= f.ncface[i]; ++k) {
      int nck = f.C(k, i);
      if (nck <= n) {
        for (int kk = 1; kk <= f.ncface[nck]; ++kk)
          if (f.C(kk, nck) == i) f.FI(f.llec, k, i) = kk;
      } else {
        int d = f.FI(f.idir, k, i);
        f.FI(f.llec, k, i) = d == 1 ? 3 : d == 3 ? 1 : d == 2 ? 4 : 2;
      }
      int d = f.FI(f.idir, k, i);
      if (d == 1 || d == 3) f.F(f.ds, k, i) = std::min(f.dx[i], f.dx[nck]);
      else f.F(f.ds, k, i) = std::min(f.dy[i], f.dy[nck]);
    }
  }
  // joint cells
  f.isjoint.assign(nD + 1, 0);
  for (int i = 1; i <= n; ++i) {
    for (int k = 1; k <= f.ncface[i]; ++k) {
      int nck = f.C(k, i);
      if (nck > n) continue;
      int d = f.FI(f.idir, k, i);
      double r = (d == 2 || d == 4) ? f.dy[i] / f.dy[nck] : f.dx[i] / f.dx[nck];
      if (r > 1.2 || r < 0.8) { f.isjoint[i] = 1; f.isjoint[nck] = 1; }
    }
  }
  f.idjoint.clear();
  for (int i = 1; i <= n; ++i)
    if (f.isjoint[i]) f.idjoint.push_back(i);
  // no-repeat face lists
  VI ind(FS, 1);
  f.nxyface.assign(nD + 1, 0); f.nxface.assign(nD + 1, 0); f.nyface.assign(nD + 1, 0);
  f.kxyface.assign(FS, 0); f.kxface.assign(FS, 0); f.kyface.assign(FS, 0);
  for (int i = 1; i <= n; ++i) {
    for (int k = 1; k <= f.ncface[i]; ++k) {
      if (ind[(size_t)i * NF + k] == 1) {
        int nck = f.C(k, i);
        ind[(size_t)i * NF + k] = 0;
        ind[(size_t)nck * NF + f.FI(f.llec, k, i)] = 0;
        f.nxyface[i]++;
        f.FI(f.kxyface, f.nxyface[i], i) = k;
        int d = f.FI(f.idir, k, i);
        if (d == 2 || d == 4) { f.nxface[i]++; f.FI(f.kxface, f.nxface[i], i) = k; }
        else { f.nyface[i]++; f.FI(f.kyface, f.nyface[i], i) = k; }
      }
    }
  }
  for (int i = 1; i <= n; ++i) {
    for (int k = 1; k <= f.ncface[i]; ++k) {
      int nck = f.C(k, i);
      double &fx = f.F(f.fnx, k, i), &fy = f.F(f.fny, k, i), &dnk = f.F(f.dn, k, i);
      double &rxx = f.F(f.rx, k, i), &ryy = f.F(f.ry, k, i);
      switch (f.FI(f.idir, k, i)) {
        case 1: fx = 0; fy = 1; dnk = std::fabs(f.y[nck] - f.y[i]); rxx = f.x[nck] - f.x[i]; ryy = f.dy[i] / 2.0; break;
        case 2: fx = 1; fy = 0; dnk = std::fabs(f.x[nck] - f.x[i]); rxx = f.dx[i] / 2.0; ryy = f.y[nck] - f.y[i]; break;
        case 3: fx = 0; fy = -1; dnk = std::fabs(f.y[nck] - f.y[i]); rxx = f.x[nck] - f.x[i]; ryy = -f.dy[i] / 2.0; break;
        default: fx = -1; fy = 0; dnk = std::fabs(f.x[nck] - f.x[i]); rxx = -f.dx[i] / 2.0; ryy = f.y[nck] - f.y[i]; break;
      }
    }
  }
  for (int i = 1; i <= n; ++i) {
    for (int k = 1; k <= f.ncface[i]; ++k) {
      double rnx = f.F(f.fnx, k, i) * std::fabs(f.F(f.rx, k, i));
      double rny = f.F(f.fny, k, i) * std::fabs(f.F(f.ry, k, i));
      f.F(f.rpx, k, i) = f.F(f.rx, k, i) - rnx;
      f.F(f.rpy, k, i) = f.F(f.ry, k, i) - rny;
      f.F(f.dsx, k, i) = f.F(f.fnx, k, i) * f.F(f.ds, k, i);
      f.F(f.dsy, k, i) = f.F(f.fny, k, i) * f.F(f.ds, k, i);
      f.F(f.dsxy, k, i) = f.F(f.ds, k, i) / f.F(f.dn, k, i);
    }
  }
  // fintp
  for (int i = 1; i <= n; ++i) {
    if (!f.isjoint[i]) {
      f.F(f.fintp, 1, i) = f.dy[i] / (f.dy[i] + f.dy[f.C(1, i)]);
      f.F(f.fintp, 2, i) = f.dx[i] / (f.dx[i] + f.dx[f.C(2, i)]);
      f.F(f.fintp, 3, i) = f.dy[i] / (f.dy[i] + f.dy[f.C(3, i)]);
      f.F(f.fintp, 4, i) = f.dx[i] / (f.dx[i] + f.dx[f.C(4, i)]);
    }
  }
  for (int i : f.idjoint) {
    for (int k = 1; k <= f.ncface[i]; ++k) {
      int nck = f.C(k, i), d = f.FI(f.idir, k, i);
      f.F(f.fintp, k, i) = (d == 2 || d == 4) ? f.dx[i] / (f.dx[i] + f.dx[nck]) : f.dy[i] / (f.dy[i] + f.dy[nck]);
    }
  }
}

// screen_weights (der_lib.f90:681-715)
void screen(int nt, const double* wxt, const double* wyt, const int* ixt, const int* iyt, int& nx, int& ny, int* ix,
            int* iy, double* wx, double* wy) {
  nx = 0; ny = 0;
  for (int k = 0; k <= nt; ++k) {
    if (std::fabs(wxt[k]) > 1.0e-8) { ++nx; ix[nx] = ixt[k]; wx[nx] = wxt[k]; }
    if (std::fabs(wyt[k]) > 1.0e-8) { ++ny; iy[ny] = iyt[k]; wy[ny] = wyt[k]; }
  }
}

// der_grad_cbgg (der_lib.f90:272-378) for cell i: Green-Gauss weights from
// the current iwet (ibc = 1 uses only wet neighbours, ibc = 0 all).
void cbgg_cell(Flow& f, Flow::GO& go, int i, int ibc) {
  const int nmf = f.nmf, nsc = go.nsc;
  if (f.iwet[i] == 0 && ibc == 1) { go.ncx[i] = 0; go.ncy[i] = 0; return; }
  std::vector<double> wx(nmf + 1, 0.0), wy(nmf + 1, 0.0);
  std::vector<int> ix(nmf + 1, 0), iy(nmf + 1, 0);
  ix[0] = i; iy[0] = i;
  for (int k = 1; k <= f.ncface[i]; ++k) {
    int nck = f.C(k, i);
    ix[k] = nck; iy[k] = nck;
    if (f.iwet[nck] == 1 || ibc == 0) {
      wx[0] = wx[0] + f.F(f.dsx, k, i) * (1.0 - f.F(f.fintp, k, i));
      wx[k] = f.F(f.dsx, k, i) * f.F(f.fintp, k, i);
      wy[0] = wy[0] + f.F(f.dsy, k, i) * (1.0 - f.F(f.fintp, k, i));
      wy[k] = f.F(f.dsy, k, i) * f.F(f.fintp, k, i);
    } else {
      wx[0] = wx[0] + f.F(f.dsx, k, i);
      wy[0] = wy[0] + f.F(f.dsy, k, i);
    }
  }
  for (int k = 0; k <= nmf; ++k) { wx[k] = wx[k] / f.areap[i]; wy[k] = wy[k] / f.areap[i]; }
  int *icx = &go.icx[(size_t)i * (nsc + 1)], *icy = &go.icy[(size_t)i * (nsc + 1)];
  double *wcx = &go.wcx[(size_t)i * (nsc + 1)], *wcy = &go.wcy[(size_t)i * (nsc + 1)];
  screen(nmf, wx.data(), wy.data(), ix.data(), iy.data(), go.ncx[i], go.ncy[i], icx, icy, wcx, wcy);
  double sx = 0, sy = 0;
  for (int q = 1; q <= go.ncx[i]; ++q) sx = sx + wcx[q];
  for (int q = 1; q <= go.ncy[i]; ++q) sy = sy + wcy[q];
  for (int q = 1; q <= go.ncx[i]; ++q) wcx[q] = wcx[q] - sx / (double)go.ncx[i];
  for (int q = 1; q <= go.ncy[i]; ++q) wcy[q] = wcy[q] - sy / (double)go.ncy[i];
}

// der_grad_cbggcr (der_lib.f90:381-443) for cell i: cell-reconstruction
// weights across refinement faces (no-repeat x and y face lists).
void cbggcr_cell(Flow& f, Flow::GO& go, int i, int ibc) {
  const int n = f.n, nmf = f.nmf, nsc = go.nsc;
  if (f.iwet[i] == 0 && ibc == 1) { go.ngx[i] = 0; go.ngy[i] = 0; return; }
  std::vector<double> gxy(nmf + 1, 0.0), gyx(nmf + 1, 0.0);
  std::vector<int> igx(nmf + 1, 0), igy(nmf + 1, 0);
  igx[0] = i; igy[0] = i;
  for (int j = 1; j <= f.nxface[i]; ++j) {
    int k = f.FI(f.kxface, j, i), nck = f.C(k, i);
    if (nck > n || std::fabs(f.dy[i] / f.dy[nck] - 1.0) < 0.1) continue;
    if (f.iwet[nck] == 0 && ibc == 1) continue;
    int jcn = f.FI(f.llec, k, i);
    gxy[0] = gxy[0] + f.F(f.dsx, k, i) * (1.0 - f.F(f.fintp, k, i)) * f.F(f.rpy, k, i) / f.areap[i];
    gxy[k] = f.F(f.dsx, k, i) * f.F(f.fintp, k, i) * f.F(f.rpy, jcn, nck) / f.areap[i];
    igx[k] = nck;
  }
  for (int j = 1; j <= f.nyface[i]; ++j) {
    int k = f.FI(f.kyface, j, i), nck = f.C(k, i);
    igy[k] = nck;
    if (nck > n || std::fabs(f.dx[i] / f.dx[nck] - 1.0) < 0.1) continue;
    if (f.iwet[nck] == 0 && ibc == 1) continue;
    int jcn = f.FI(f.llec, k, i);
    gyx[0] = gyx[0] + f.F(f.dsy, k, i) * (1.0 - f.F(f.fintp, k, i)) * f.F(f.rpx, k, i) / f.areap[i];
    gyx[k] = f.F(f.dsy, k, i) * f.F(f.fintp, k, i) * f.F(f.rpx, jcn, nck) / f.areap[i];
  }
  screen(nmf, gxy.data(), gyx.data(), igx.data(), igy.data(), go.ngx[i], go.ngy[i],
         &go.igx[(size_t)i * (nsc + 1)], &go.igy[(size_t)i * (nsc + 1)], &go.wgxy[(size_t)i * (nsc + 1)],
         &go.wgyx[(size_t)i * (nsc + 1)]);
}

// der_init's operator build (derivatives.f90:95-150) for the current iwet:
// cbgg for every cell, cbggcr for the joint cells (its weights are zero
// elsewhere on these grids, and der_grad_eval applies them to joint cells only).
void build_go(Flow& f, Flow::GO& go, int ibc) {
  const int n = f.n, nD = f.nD, nmf = f.nmf;
  go.nsc = nmf + 1;  // room for the cell and every face (derivatives.f90:125-131 sizes it the same or larger)
  const int nsc = go.nsc;
  go.ncx.assign(nD + 1, 0); go.ncy.assign(nD + 1, 0);
  go.icx.assign((size_t)(nD + 1) * (nsc + 1), 0); go.icy = go.icx;
  go.wcx.assign((size_t)(nD + 1) * (nsc + 1), 0.0); go.wcy = go.wcx;
  go.ngx.assign(nD + 1, 0); go.ngy.assign(nD + 1, 0);
  go.igx = go.icx; go.igy = go.icx; go.wgxy = go.wcx; go.wgyx = go.wcx;
  go.ider = (f.skewcor && !f.idjoint.empty()) ? 2 : 1;
  for (int i = 1; i <= n; ++i) cbgg_cell(f, go, i, ibc);
  if (go.ider != 2) return;
  for (int i : f.idjoint) cbggcr_cell(f, go, i, ibc);
}

// der_update (derivatives.f90:204-296): the wet-cell operator is recomputed
// for every active cell whose wet state differs from the previous time level
// and for its neighbours.  Only active cells' changes are looked at; a dummy
// whose state changes does not flag its cell.
int der_update(Flow& f) {
  const int n = f.n;
  std::vector<char> ichg(f.nD + 1, 0);
  for (int i = 1; i <= n; ++i)
    if (f.iwet[i] != f.iwet1[i]) {
      ichg[i] = 1;
      for (int k = 1; k <= f.ncface[i]; ++k) ichg[f.C(k, i)] = 1;
    }
  int nlist = 0;
  for (int i = 1; i <= n; ++i) {
    if (!ichg[i]) continue;
    ++nlist;
    cbgg_cell(f, f.gow, i, 1);
    if (f.gow.ider == 2) cbggcr_cell(f, f.gow, i, 1);
  }
  return nlist;
}

// flow_pond (flow.F90:1807-1876): wet cells not connected through wet cells
// to a forcing-boundary string are dried.  The string cells and their dummies
// seed the search; the alternating forward/backward sweeps run until a pass
// adds nothing.
void flow_pond(Flow& f) {
  const int n = f.n, nD = f.nD;
  std::vector<int> ipond(nD + 1, 0);
  for (size_t j = 0; j < f.th_cells.size(); ++j) {
    const int i = f.th_cells[j], k = f.th_faces[j];
    ipond[i] = f.iwet[i];
    const int nck = f.C(k, i);
    ipond[nck] = f.iwet[nck];
  }
  int npond = 10;
  while (npond > 0) {
    npond = 0;
    for (int i = 1; i <= n; ++i) {
      if (ipond[i] != 1) continue;
      for (int k = 1; k <= f.ncface[i]; ++k) {
        const int nck = f.C(k, i);
        npond = npond + std::max(0, f.iwet[nck] - ipond[nck]);
        ipond[nck] = f.iwet[nck];
      }
    }
    for (int i = n; i >= 1; --i) {
      if (ipond[i] != 1) continue;
      for (int k = 1; k <= f.ncface[i]; ++k) {
        const int nck = f.C(k, i);
        npond = npond + std::max(0, f.iwet[nck] - ipond[nck]);
        ipond[nck] = f.iwet[nck];
      }
    }
  }
  for (int i = 1; i <= nD; ++i)
    if (ipond[i] == 0 && f.iwet[i] == 1) f.iwet[i] = 0;
}

// flow_wetdry(0) (flow.F90:1231-1539) for Cartesian and telescoping grids
// (ncellpoly = 0) without structures: depth rule, closed-boundary dummies dry,
// narrow-channel removal (narrowchannels off) or the one-cell rule
// (narrowchannels on), flow_pond (ponding off), corner cells, dry-to-wet
// initialisation (5 passes, in cell order), and zero flux and viscosity on
// every face with a dry side.
void flow_wetdry(Flow& f) {
  const Params& P = f.P;
  const int n = f.n, nD = f.nD;
  const double gravinv = 1.0 / P.grav;
  for (int i = 1; i <= nD; ++i) {
    f.h[i] = f.p[i] * gravinv - f.zb[i];
    if (f.h[i] < P.hdry) {
      f.h[i] = std::max(f.h[i], P.hmin);
      f.iwet[i] = 0;
    } else {
      f.iwet[i] = 1;
    }
  }
  for (size_t j = 0; j < f.w_cells.size(); ++j) f.iwet[f.C(f.w_faces[j], f.w_cells[j])] = 0;
  auto dir = [&](int k, int i) { return f.FI(f.idir, k, i); };
  if (P.narrowchannels) {
    int nsw = 1;
    while (nsw > 0) {
      nsw = 0;
      for (int i = 1; i <= n; ++i) {
        if (f.iwet[i] == 0) continue;
        int ksum = 0;
        for (int k = 1; k <= f.ncface[i]; ++k) ksum += f.iwet[f.C(k, i)];
        if (ksum == 0) { f.iwet[i] = 0; ++nsw; }
      }
    }
  } else {
    int nsw = 1;
    while (nsw > 0) {
      nsw = 0;
      for (int i = 1; i <= n; ++i) {
        if (f.iwet[i] == 0) continue;
        int ksum = 0;
        for (int k = 1; k <= f.ncface[i]; ++k) ksum += f.iwet[f.C(k, i)];
        if (ksum <= 1) { f.iwet[i] = 0; ++nsw; }
        int kns = 0, kew = 0;
        for (int k = 1; k <= f.ncface[i]; ++k) {
          const int nck = f.C(k, i), d = dir(k, i);
          if (d == 1 || d == 3) kns += f.iwet[nck];
          if (d == 2 || d == 4) kew += f.iwet[nck];
        }
        if ((kns == 0 || kew == 0) && f.h[i] < P.hdry1) { f.iwet[i] = 0; ++nsw; }
        // a direct neighbour on side a plus the cells beyond the neighbour on side b
        auto pair_sum = [&](int a, int b) {
          int s = 0;
          for (int k = 1; k <= f.ncface[i]; ++k) {
            const int nck = f.C(k, i);
            if (dir(k, i) == a) s += f.iwet[nck];
            if (dir(k, i) == b)
              for (int kk = 1; kk <= f.ncface[nck]; ++kk)
                if (dir(kk, nck) == b) s += f.iwet[f.C(kk, nck)];
          }
          return s;
        };
        const int knss = pair_sum(1, 3);
        if (knss == 0 && f.h[i] < P.hdry2) { f.iwet[i] = 0; ++nsw; }
        // the north-north count (flow.F90:1384-1392) is formed but the test
        // that follows reads knss again (flow.F90:1394)
        if (knss == 0 && f.h[i] < P.hdry2) { f.iwet[i] = 0; ++nsw; }
        const int keww = pair_sum(2, 4);
        if (keww == 0 && f.h[i] < P.hdry2) { f.iwet[i] = 0; ++nsw; }
        const int keew = pair_sum(4, 2);
        if (keew == 0 && f.h[i] < P.hdry2) { f.iwet[i] = 0; ++nsw; }
      }
    }
  }
  if (!P.ponding) flow_pond(f);
  for (int i = 1; i <= n; ++i) {
    f.icorner[i] = 0;
    if (f.iwet[i] == 1) {
      int nd = 0;
      for (int k = 1; k <= f.ncface[i]; ++k) if (f.iwet[f.C(k, i)] == 0) ++nd;
      if (nd > 1) f.icorner[i] = 1;
    }
  }
  for (int pass = 0; pass < 5; ++pass)
    for (int i = 1; i <= n; ++i) {
      if (!(f.iwet[i] == 1 && f.iwet1[i] == 0)) continue;
      double us = 0, vs = 0, viss = 0;
      int ns = 0;
      for (int k = 1; k <= f.ncface[i]; ++k) {
        const int nck = f.C(k, i);
        us = us + f.u[nck]; vs = vs + f.v[nck]; viss = viss + f.vis[nck]; ns += f.iwet[nck];
      }
      f.u[i] = us / ((double)ns + P.small) / 1.25;
      f.v[i] = vs / ((double)ns + P.small) / 1.25;
      f.vis[i] = viss / ((double)ns + P.small);
    }
  for (int i = 1; i <= n; ++i)
    for (int j = 1; j <= f.nxyface[i]; ++j) {
      const int k = f.FI(f.kxyface, j, i), nck = f.C(k, i), jcn = f.FI(f.llec, k, i);
      if (f.iwet[i] * f.iwet[nck] == 0) {
        f.F(f.flux, k, i) = 0.0; f.F(f.visk, k, i) = 0.0;
        f.F(f.flux, jcn, nck) = 0.0; f.F(f.visk, jcn, nck) = 0.0;
      }
    }
}

// The solver's residual weights follow iwet (natural and permuted solvers).
void solver_set_wet(Flow& f) {
  const int n = f.n, nD = f.nD;
  std::vector<int> iw(nD);
  for (int i = 1; i <= nD; ++i) iw[i - 1] = f.iwet[i];
  orc_set_wet(f.solver, iw.data());
  if (f.solver_perm) {
    for (int r = 0; r < nD; ++r) iw[r] = f.iwet[(r < n ? f.perm[r] : r) + 1];
    orc_set_wet(f.solver_perm, iw.data());
  }
}

// der_grad_eval (der_lib.f90:726-842), ilim = 0.
void grad_eval(Flow& f, Flow::GO& go, const V& var, V& dvx, V& dvy) {
  const int nsc1 = go.nsc + 1;
  V xm, ym;
  if (go.ider == 2) { xm = dvx; ym = dvy; }
  for (int i = 1; i <= f.n; ++i) {
    double a = 0;
    for (int q = 1; q <= go.ncx[i]; ++q) a = a + go.wcx[(size_t)i * nsc1 + q] * var[go.icx[(size_t)i * nsc1 + q]];
    dvx[i] = a;
    a = 0;
    for (int q = 1; q <= go.ncy[i]; ++q) a = a + go.wcy[(size_t)i * nsc1 + q] * var[go.icy[(size_t)i * nsc1 + q]];
    dvy[i] = a;
  }
  if (go.ider == 2) {
    for (int i : f.idjoint) {
      for (int q = 1; q <= go.ngx[i]; ++q) dvx[i] = dvx[i] + go.wgxy[(size_t)i * nsc1 + q] * ym[go.igx[(size_t)i * nsc1 + q]];
      for (int q = 1; q <= go.ngy[i]; ++q) dvy[i] = dvy[i] + go.wgyx[(size_t)i * nsc1 + q] * xm[go.igy[(size_t)i * nsc1 + q]];
    }
  }
}

// der_gradvec_eval (der_lib.f90:936-1049), ilim = 0.
void gradvec_eval(Flow& f, Flow::GO& go, const V& u, const V& v, V& dux, V& duy, V& dvx, V& dvy) {
  const int nsc1 = go.nsc + 1;
  V uxm, uym, vxm, vym;
  if (go.ider == 2) { uxm = dux; uym = duy; vxm = dvx; vym = dvy; }
  for (int i = 1; i <= f.n; ++i) {
    double a = 0, b = 0;
    for (int q = 1; q <= go.ncx[i]; ++q) {
      int nck = go.icx[(size_t)i * nsc1 + q];
      a = a + go.wcx[(size_t)i * nsc1 + q] * u[nck];
      b = b + go.wcx[(size_t)i * nsc1 + q] * v[nck];
    }
    dux[i] = a; dvx[i] = b;
    a = 0; b = 0;
    for (int q = 1; q <= go.ncy[i]; ++q) {
      int nck = go.icy[(size_t)i * nsc1 + q];
      a = a + go.wcy[(size_t)i * nsc1 + q] * u[nck];
      b = b + go.wcy[(size_t)i * nsc1 + q] * v[nck];
    }
    duy[i] = a; dvy[i] = b;
  }
  if (go.ider == 2) {
    for (int i : f.idjoint) {
      for (int q = 1; q <= go.ngx[i]; ++q) {
        int nck = go.igx[(size_t)i * nsc1 + q];
        double w = go.wgxy[(size_t)i * nsc1 + q];
        dux[i] = dux[i] + w * uym[nck];
        dvx[i] = dvx[i] + w * vym[nck];
      }
      for (int q = 1; q <= go.ngy[i]; ++q) {
        int nck = go.igy[(size_t)i * nsc1 + q];
        double w = go.wgyx[(size_t)i * nsc1 + q];
        duy[i] = duy[i] + w * uxm[nck];
        dvy[i] = dvy[i] + w * vxm[nck];
      }
    }
  }
}

// interp_scal_cell2face (interp_lib.f90:2727-2906) for ibc = 0, 1, 3 with the
// skewness correction for joint cells when gradients are given.
void interp_c2f(Flow& f, const V& phi, int ibc, V& phik, const V* dphix, const V* dphiy) {
  for (int i = 1; i <= f.n; ++i) {
    for (int j = 1; j <= f.nxyface[i]; ++j) {
      int k = f.FI(f.kxyface, j, i), nck = f.C(k, i), jcn = f.FI(f.llec, k, i);
      double fk = f.F(f.fintp, k, i), val;
      if (ibc == 0) {
        val = fk * phi[nck] + (1.0 - fk) * phi[i];
      } else if (ibc == 1) {
        if (f.iwet[i] * f.iwet[nck] == 1) val = fk * phi[nck] + (1.0 - fk) * phi[i];
        else if (f.iwet[i] == 1) val = phi[i];
        else if (f.iwet[nck] == 1) val = phi[nck];
        else val = 0.5 * (phi[i] + phi[nck]);
      } else {  // 3
        val = (f.iwet[i] * f.iwet[nck] == 1) ? fk * phi[nck] + (1.0 - fk) * phi[i] : 0.0;
      }
      f.F(phik, k, i) = val;
      f.F(phik, jcn, nck) = val;
    }
  }
  if (f.skewcor && dphiy) {
    for (int i : f.idjoint) {
      for (int j = 1; j <= f.nxyface[i]; ++j) {
        int k = f.FI(f.kxyface, j, i), nck = f.C(k, i), jcn = f.FI(f.llec, k, i);
        double fk = f.F(f.fintp, k, i);
        double& pkv = f.F(phik, k, i);
        if (std::fabs(f.F(f.fnx, k, i)) > 0.999)
          pkv = pkv + fk * f.F(f.rpy, jcn, nck) * (*dphiy)[nck] + (1.0 - fk) * f.F(f.rpy, k, i) * (*dphiy)[i];
        else
          pkv = pkv + fk * f.F(f.rpx, jcn, nck) * (*dphix)[nck] + (1.0 - fk) * f.F(f.rpx, k, i) * (*dphix)[i];
        pkv = std::min(std::max(pkv, std::min(phi[i], phi[nck])), std::max(phi[i], phi[nck]));
        f.F(phik, jcn, nck) = pkv;
      }
    }
  }
}

// flow_grad_interp (flow_imp.F90:1075-1130)
void flow_grad_interp(Flow& f) {
  gradvec_eval(f, f.gow, f.u, f.v, f.dux, f.duy, f.dvx, f.dvy);
  interp_c2f(f, f.p, 1, f.pk, &f.dpx, &f.dpy);
  const double gravinv = 1.0 / f.P.grav;
  for (int i = 1; i <= f.n; ++i) {
    double ax = 0, ay = 0;
    for (int k = 1; k <= f.ncface[i]; ++k) {
      ax = ax + f.F(f.dsx, k, i) * f.F(f.pk, k, i);
      ay = ay + f.F(f.dsy, k, i) * f.F(f.pk, k, i);
      f.F(f.hk, k, i) = std::max(f.P.hmin, f.F(f.pk, k, i) * gravinv - f.F(f.zbk, k, i));
    }
    f.dpx[i] = ax / f.areap[i];
    f.dpy[i] = ay / f.areap[i];
  }
}

// fric_eval (friction.F90:615-797): Manning (mbedfric 2), no waves.
void fric_eval(Flow& f) {
  const double g = f.P.grav;
  for (int i = 1; i <= f.n; ++i) {
    f.cfrict[i] = man2drag(g, f.coefman[i], f.h[i], 10.0);
    if (f.cfrict[i] != 0.0) f.z0[i] = drag2length(f.cfrict[i], f.h[i]);
  }
  for (int i = 1; i <= f.n; ++i) {  // fric_curmean_quad, fric_lib.f90:877-905 (rhow cancels)
    double um = std::sqrt(f.u[i] * f.u[i] + f.v[i] * f.v[i]);
    f.uv[i] = um;
    f.uelwc[i] = um;
    double taum = 1025.0 * f.cfrict[i] * um * um;
    f.bsxy[i] = taum;
    f.bsvel[i] = std::sqrt(taum / 1025.0 + 1.0e-15);
  }
}

// flow_eddyvis, mturbul = 5 without waves (flow_eddyvis.f90:136-222)
void flow_eddyvis(Flow& f) {
  const Params& P = f.P;
  for (int i = 1; i <= f.n; ++i) {
    if (f.iwet[i] == 1) {
      double st = std::sqrt(2.0 * (f.dux[i] * f.dux[i] + f.dvy[i] * f.dvy[i]) + (f.duy[i] + f.dvx[i]) * (f.duy[i] + f.dvx[i]));
      double vi = P.cviscon + P.cvisbot * f.bsvel[i] * f.h[i] + f.cvishor2areaavg * st;
      f.vis[i] = std::min(vi, P.cvismax);
    } else {
      f.vis[i] = 1.0e-6;
    }
  }
  // bndcopy2ghost (boundaries.F90:4417-4437): open-boundary strings
  for (size_t j = 0; j < f.th_cells.size(); ++j) f.vis[f.C(f.th_faces[j], f.th_cells[j])] = f.vis[f.th_cells[j]];
  static const int kkface[5] = {0, 3, 4, 1, 2};
  for (int i = 1; i <= f.n; ++i) {
    if (f.iwet[i] != 1) continue;
    for (int k = 1; k <= f.ncface[i]; ++k) {
      int nck = f.C(k, i);
      if (f.iwet[nck] == 0 || nck > f.n) {
        int kkdf = kkface[f.FI(f.idir, k, i)];
        double cid = 0, vs = 0;
        for (int kk = 1; kk <= f.ncface[i]; ++kk)
          if (f.FI(f.idir, kk, i) == kkdf) { cid = cid + 1.0; vs = vs + f.vis[f.C(kk, i)] - P.cviscon; }
        f.vis[i] = P.cviscon + vs / (cid + 1.0e-15);
        f.vis[nck] = f.vis[i];
      }
    }
  }
  for (int i = 1; i <= f.n; ++i) {
    if (f.icorner[i] == 1) {
      double cid = 0, vs = 0;
      for (int k = 1; k <= f.ncface[i]; ++k) {
        int nck = f.C(k, i);
        cid = cid + f.iwet[nck];
        vs = vs + (f.vis[nck] - P.cviscon) * f.iwet[nck];
      }
      f.vis[i] = P.cviscon + vs / (cid + 1.0e-15);
    }
  }
  interp_c2f(f, f.vis, 3, f.visk, nullptr, nullptr);
}

// flow_srcsnk_static, ntsch = 1 (flow_imp.F90:336-346)
void srcsnk_static(Flow& f, double dt) {
  const double gdi = 1.0 / (f.P.grav * dt), dti = 1.0 / dt;
  for (int i = 1; i <= f.n; ++i) {
    double fac1 = f.areap[i] * f.h1[i] * dti;
    f.spuv0[i] = -fac1;
    f.ssu0[i] = fac1 * f.u1[i];
    f.ssv0[i] = fac1 * f.v1[i];
    f.sppp0[i] = -f.areap[i] * gdi;
    f.sspp0[i] = -f.p1[i] * f.sppp0[i];
  }
}

// coeffsourcesink_uv(schemecoef) (flow_imp.F90:409-466)
void coef_uv(Flow& f) {
  for (int i = 1; i <= f.n; ++i) {
    f.su[i] = f.ssu0[i] + (f.fc[i] * f.v[i] - f.dpx[i]) * f.h[i] * f.areap[i];
    f.sv[i] = f.ssv0[i] + (-f.fc[i] * f.u[i] - f.dpy[i]) * f.h[i] * f.areap[i];
    f.cbcfuwcap[i] = f.cmb[i] * f.cfrict[i] * f.uelwc[i] * f.areap[i];
    f.sp[i] = f.spuv0[i] - f.cbcfuwcap[i];
    for (int k = 1; k <= f.ncface[i]; ++k) {
      double ddk = f.F(f.visk, k, i) * f.F(f.hk, k, i) * f.F(f.dsxy, k, i);
      f.F(f.acoef, k, i) = schemecoef(f.P.ndsch, ddk, f.F(f.flux, k, i));
    }
  }
}

// defcorparagradvec (computational.F90:149-264), joint cells
void defcor(Flow& f) {
  V uskew((size_t)(f.nD + 1) * f.NF, 0.0), vskew = uskew;
  for (int i : f.idjoint) {
    if (f.iwet[i] == 0) continue;
    for (int j = 1; j <= f.nxface[i]; ++j) {
      int k = f.FI(f.kxface, j, i), nck = f.C(k, i);
      if (nck > f.n || f.iwet[nck] == 0) continue;
      int jcn = f.FI(f.llec, k, i);
      if (std::fabs(f.F(f.rpy, k, i)) > 1.0e-6) {
        double val = (f.F(f.acoef, k, i) + f.F(f.flux, k, i)) * f.F(f.rpy, k, i);
        f.F(uskew, k, i) = val * f.duy[i]; f.F(vskew, k, i) = val * f.dvy[i];
        f.F(uskew, jcn, nck) = -f.F(uskew, k, i); f.F(vskew, jcn, nck) = -f.F(vskew, k, i);
      } else if (std::fabs(f.F(f.rpy, jcn, nck)) > 1.0e-6) {
        double val = -f.F(f.acoef, k, i) * f.F(f.rpy, jcn, nck);
        f.F(uskew, k, i) = val * f.duy[nck]; f.F(vskew, k, i) = val * f.dvy[nck];
        f.F(uskew, jcn, nck) = -f.F(uskew, k, i); f.F(vskew, jcn, nck) = -f.F(vskew, k, i);
      }
    }
    for (int j = 1; j <= f.nyface[i]; ++j) {
      int k = f.FI(f.kyface, j, i), nck = f.C(k, i);
      if (nck > f.n || f.iwet[nck] == 0) continue;
      int jcn = f.FI(f.llec, k, i);
      if (std::fabs(f.F(f.rpx, k, i)) > 1.0e-6) {
        double val = (f.F(f.acoef, k, i) + f.F(f.flux, k, i)) * f.F(f.rpx, k, i);
        f.F(uskew, k, i) = val * f.dux[i]; f.F(vskew, k, i) = val * f.dvx[i];
        f.F(uskew, jcn, nck) = -f.F(uskew, k, i); f.F(vskew, jcn, nck) = -f.F(vskew, k, i);
      } else if (std::fabs(f.F(f.rpx, jcn, nck)) > 1.0e-6) {
        double val = -f.F(f.acoef, k, i) * f.F(f.rpx, jcn, nck);
        f.F(uskew, k, i) = val * f.dux[nck]; f.F(vskew, k, i) = val * f.dvx[nck];
        f.F(uskew, jcn, nck) = -f.F(uskew, k, i); f.F(vskew, jcn, nck) = -f.F(vskew, k, i);
      }
    }
  }
  for (int i : f.idjoint) {
    double a = 0, b = 0;
    for (int k = 1; k <= f.ncface[i]; ++k) { a = a + f.F(uskew, k, i); b = b + f.F(vskew, k, i); }
    f.su[i] = f.su[i] - a;
    f.sv[i] = f.sv[i] - b;
  }
}

// bound_uv (boundaries.F90:3310-3490) with TH strings (bnd_vel_openwse,
// bnd_vel.f90:35-95) and wall friction (wallfric = .true.)
void bound_uv(Flow& f) {
  for (size_t j = 0; j < f.th_cells.size(); ++j) {
    int i = f.th_cells[j], k = f.th_faces[j], nck = f.C(k, i);
    double ddk = f.F(f.visk, k, i) * f.F(f.hk, k, i) * f.F(f.dsxy, k, i);
    double a = upwindcoef(ddk, f.F(f.flux, k, i));
    f.F(f.acoef, k, i) = a;
    if (std::fabs(f.F(f.fny, k, i)) > 0.9999) {
      f.u[nck] = f.iwet[i] * f.u[i] * f.h[i] / f.h[nck];
      f.v[nck] = f.F(f.fny, k, i) * f.F(f.flux, k, i) / (f.F(f.ds, k, i) * f.F(f.hk, k, i));
      f.sv[i] = f.sv[i] + a * f.v[nck];
    } else {
      f.u[nck] = f.F(f.fnx, k, i) * f.F(f.flux, k, i) / (f.F(f.ds, k, i) * f.F(f.hk, k, i));
      f.v[nck] = f.iwet[i] * f.v[i] * f.h[i] / f.h[nck];
      f.su[i] = f.su[i] + a * f.u[nck];
    }
    f.sp[i] = f.sp[i] - a;
    f.F(f.acoef, k, i) = 0.0;
  }
  for (int i = 1; i <= f.n; ++i) {
    if (f.iwet[i] == 1) {
      f.spu[i] = f.sp[i];
      f.spv[i] = f.sp[i];
      for (int k = 1; k <= f.ncface[i]; ++k) {
        int nck = f.C(k, i);
        if (f.iwet[nck] == 0) {
          double z0wall = f.z0[i] * f.P.wallfac;
          if (std::fabs(f.F(f.fny, k, i)) > 0.999) {
            double delta = std::fabs(f.F(f.ry, k, i));
            f.spu[i] = f.spu[i] - f.F(f.ds, k, i) * f.F(f.hk, k, i) * wall_coef(delta, z0wall) * std::fabs(f.u[i]);
          } else {
            double delta = std::fabs(f.F(f.rx, k, i));
            f.spv[i] = f.spv[i] - f.F(f.ds, k, i) * f.F(f.hk, k, i) * wall_coef(delta, z0wall) * std::fabs(f.v[i]);
          }
        }
      }
    } else {
      f.u[i] = 0.0; f.v[i] = 0.0;
      f.spu[i] = -1.0; f.spv[i] = -1.0; f.sp[i] = -1.0;
      f.su[i] = 0.0; f.sv[i] = 0.0;
    }
  }
}

// flow_imp_flux_skew / _noskew (flow_imp_flux.f90:2-169, 361-409)
void flux_eval(Flow& f) {
  const int n = f.n;
  if (!f.skewcor) {
    for (int i = 1; i <= n; ++i) {
      for (int j = 1; j <= f.nxyface[i]; ++j) {
        int k = f.FI(f.kxyface, j, i), nck = f.C(k, i);
        double fl;
        if (f.iwet[i] * f.iwet[nck] == 0) fl = 0.0;
        else if (nck > n)
          fl = f.F(f.hk, k, i) * f.F(f.ds, k, i) * ((f.F(f.fnx, k, i) * f.Hu[i] + f.F(f.fny, k, i) * f.Hv[i]) -
               f.apuareap[i] * f.F(f.hk, k, i) * (f.p[nck] - f.p[i]) / f.F(f.dn, k, i));
        else {
          double fk = f.F(f.fintp, k, i), fp = 1.0 - fk;
          double ap = fk * f.apuareap[nck] + fp * f.apuareap[i];
          double huf = fk * f.Hu[nck] + fp * f.Hu[i], hvf = fk * f.Hv[nck] + fp * f.Hv[i];
          fl = f.F(f.hk, k, i) * f.F(f.ds, k, i) * ((f.F(f.fnx, k, i) * huf + f.F(f.fny, k, i) * hvf) -
               ap * f.F(f.hk, k, i) * (f.p[nck] - f.p[i]) / f.F(f.dn, k, i));
        }
        f.F(f.flux, k, i) = fl;
        f.F(f.flux, f.FI(f.llec, k, i), nck) = -fl;
      }
    }
    return;
  }
  gradvec_eval(f, f.gow, f.Hu, f.Hv, f.dHux, f.dHuy, f.dHvx, f.dHvy);
  grad_eval(f, f.gow, f.apuareap, f.dapx, f.dapy);
  for (int i = 1; i <= n; ++i) {
    const bool joint = f.isjoint[i];
    for (int pass = 0; pass < 2; ++pass) {  // x faces then y faces
      const int nf = pass == 0 ? f.nxface[i] : f.nyface[i];
      for (int j = 1; j <= nf; ++j) {
        int k = pass == 0 ? f.FI(f.kxface, j, i) : f.FI(f.kyface, j, i);
        int nck = f.C(k, i), jcn = f.FI(f.llec, k, i);
        const double fn = pass == 0 ? f.F(f.fnx, k, i) : f.F(f.fny, k, i);
        const V& H = pass == 0 ? f.Hu : f.Hv;
        double fl;
        if (f.iwet[i] * f.iwet[nck] == 0) fl = 0.0;
        else if (nck > n)
          fl = f.F(f.hk, k, i) * f.F(f.ds, k, i) * (fn * H[i] - f.apuareap[i] * f.F(f.hk, k, i) * (f.p[nck] - f.p[i]) / f.F(f.dn, k, i));
        else {
          double fk = f.F(f.fintp, k, i), fp = 1.0 - fk, ap, hf, dpf;
          if (!joint) {
            ap = fk * f.apuareap[nck] + fp * f.apuareap[i];
            hf = fk * H[nck] + fp * H[i];
            fl = f.F(f.hk, k, i) * f.F(f.ds, k, i) * (fn * hf - ap * f.F(f.hk, k, i) * (f.p[nck] - f.p[i]) / f.F(f.dn, k, i));
          } else {
            // x faces use rpy/dHuy/dapy/dpy; y faces rpx/dHvx/dapx/dpx
            const double rpk = pass == 0 ? f.F(f.rpy, k, i) : f.F(f.rpx, k, i);
            const double rpn = pass == 0 ? f.F(f.rpy, jcn, nck) : f.F(f.rpx, jcn, nck);
            const V& dap = pass == 0 ? f.dapy : f.dapx;
            const V& dH = pass == 0 ? f.dHuy : f.dHvx;
            const V& dp = pass == 0 ? f.dpy : f.dpx;
            if (std::fabs(rpk) > 1.0e-6) {
              ap = fk * f.apuareap[nck] + fp * (f.apuareap[i] + rpk * dap[i]);
              hf = fk * H[nck] + fp * (H[i] + rpk * dH[i]);
              dpf = (f.p[nck] - f.p[i] - rpk * dp[i]) / f.F(f.dn, k, i);
            } else if (std::fabs(rpn) > 1.0e-6) {
              ap = fk * (f.apuareap[nck] + rpn * dap[nck]) + fp * f.apuareap[i];
              hf = fk * (H[nck] + rpn * dH[nck]) + fp * H[i];
              dpf = (f.p[nck] + rpn * dp[nck] - f.p[i]) / f.F(f.dn, k, i);
            } else {
              ap = fk * f.apuareap[nck] + fp * f.apuareap[i];
              hf = fk * H[nck] + fp * H[i];
              dpf = (f.p[nck] - f.p[i]) / f.F(f.dn, k, i);
            }
            fl = f.F(f.hk, k, i) * f.F(f.ds, k, i) * (fn * hf - ap * f.F(f.hk, k, i) * dpf);
          }
        }
        f.F(f.flux, k, i) = fl;
        f.F(f.flux, jcn, nck) = -fl;
      }
    }
  }
}

// coefsourcesink_pp (flow_imp.F90:577-794), ntsch = 1
void coef_pp(Flow& f) {
  const int n = f.n;
  for (int i = 1; i <= n; ++i) {
    double asum = 0;
    for (int k = 1; k <= f.ncface[i]; ++k) asum = asum + f.F(f.acoef, k, i);
    double apu = f.iwet[i] * f.P.relax_uv / std::max(asum - f.sp[i], 1.0e-6);
    f.apuareap[i] = apu * f.areap[i];
    f.sumu[i] = asum * apu;
    f.Hu[i] = f.iwet[i] * (f.u[i] + f.apuareap[i] * f.dpx[i] * f.h[i]);
    f.Hv[i] = f.iwet[i] * (f.v[i] + f.apuareap[i] * f.dpy[i] * f.h[i]);
  }
  for (int i = 1; i <= n; ++i) {
    for (int j = 1; j <= f.nxyface[i]; ++j) {
      int k = f.FI(f.kxyface, j, i), nck = f.C(k, i);
      double a;
      if (f.iwet[i] * f.iwet[nck] == 0) a = 0.0;
      else if (nck > n)
        a = f.F(f.hk, k, i) * f.F(f.hk, k, i) * f.F(f.ds, k, i) * f.apuareap[i] / (1.0 - f.sumu[i]) / f.F(f.dn, k, i);
      else {
        double fk = f.F(f.fintp, k, i), fp = 1.0 - fk;
        double apv = fk * f.apuareap[nck] + fp * f.apuareap[i];
        double suf = fk * f.sumu[nck] + fp * f.sumu[i];
        a = f.F(f.hk, k, i) * f.F(f.hk, k, i) * f.F(f.ds, k, i) * apv / (1.0 - suf) / f.F(f.dn, k, i);
      }
      f.F(f.acoef, k, i) = a;
      f.F(f.acoef, f.FI(f.llec, k, i), nck) = a;
    }
  }
  flux_eval(f);
  for (int i = 1; i <= n; ++i) {
    f.sp[i] = f.sppp0[i];
    double s = 0;
    for (int k = 1; k <= f.ncface[i]; ++k) s = s + f.F(f.flux, k, i);
    f.su[i] = f.sspp0[i] - s + f.p[i] * f.sp[i];
  }
  if (f.skewcor && !f.idjoint.empty()) {
    V fcorr((size_t)(f.nD + 1) * f.NF, 0.0);
    for (int i : f.idjoint) {
      if (f.iwet[i] == 0) continue;
      for (int j = 1; j <= f.nxface[i]; ++j) {
        int k = f.FI(f.kxface, j, i), nck = f.C(k, i);
        if (f.iwet[nck] == 0) continue;
        int jcn = f.FI(f.llec, k, i);
        if (std::fabs(f.F(f.rpy, k, i)) > 1.0e-6) {
          f.F(fcorr, k, i) = -f.F(f.acoef, k, i) * f.F(f.rpy, k, i) * f.dppy[i];
          f.F(fcorr, jcn, nck) = -f.F(fcorr, k, i);
        } else if (std::fabs(f.F(f.rpy, jcn, nck)) > 1.0e-6) {
          f.F(fcorr, k, i) = f.F(f.acoef, k, i) * f.F(f.rpy, jcn, nck) * f.dppy[nck];
          f.F(fcorr, jcn, nck) = -f.F(fcorr, k, i);
        }
      }
      for (int j = 1; j <= f.nyface[i]; ++j) {
        int k = f.FI(f.kyface, j, i), nck = f.C(k, i);
        if (f.iwet[nck] == 0) continue;
        int jcn = f.FI(f.llec, k, i);
        if (std::fabs(f.F(f.rpx, k, i)) > 1.0e-6) {
          f.F(fcorr, k, i) = -f.F(f.acoef, k, i) * f.F(f.rpx, k, i) * f.dppx[i];
          f.F(fcorr, jcn, nck) = -f.F(fcorr, k, i);
        } else if (std::fabs(f.F(f.rpx, jcn, nck)) > 1.0e-6) {
          f.F(fcorr, k, i) = f.F(f.acoef, k, i) * f.F(f.rpx, jcn, nck) * f.dppx[nck];
          f.F(fcorr, jcn, nck) = -f.F(fcorr, k, i);
        }
      }
    }
    for (int i : f.idjoint) {
      double s = 0;
      for (int k = 1; k <= f.ncface[i]; ++k) s = s + f.F(fcorr, k, i);
      f.su[i] = f.su[i] + 0.2 * s;
    }
  }
}

// bound_pp (boundaries.F90:3493-3646) with bnd_pp (4767-4795) for the TH strings
void bound_pp(Flow& f) {
  for (int i = 1; i <= f.n; ++i) {
    if (f.iwet[i] != 0) continue;
    int sumwet = 0;
    for (int k = 1; k <= f.ncface[i]; ++k) { int nck = f.C(k, i); if (nck <= f.n) sumwet += f.iwet[nck]; }
    double aploc = 0;
    f.su[i] = 0.0;
    for (int k = 1; k <= f.ncface[i]; ++k) {
      int nck = f.C(k, i);
      if (sumwet >= 1) { f.F(f.acoef, k, i) = f.iwet[nck]; }
      else if (nck > f.n) { f.F(f.acoef, k, i) = 0.0; continue; }
      else f.F(f.acoef, k, i) = f.F(f.dsxy, k, i);
      aploc = aploc + f.F(f.acoef, k, i);
      f.su[i] = f.su[i] + f.F(f.acoef, k, i) * f.p[nck];
    }
    f.su[i] = f.su[i] - aploc * f.p[i];
    f.sp[i] = 0.0;
  }
  for (size_t j = 0; j < f.th_cells.size(); ++j) {
    int i = f.th_cells[j], k = f.th_faces[j], nck = f.C(k, i);
    f.pp[nck] = f.wsebnd[j] * f.P.grav - f.p[nck];
    f.su[i] = f.su[i] + f.F(f.acoef, k, i) * f.pp[nck];
    f.sp[i] = f.sp[i] - f.F(f.acoef, k, i);
    f.F(f.acoef, k, i) = 0.0;
  }
}

// pvfc (flow_imp.F90:797-1072)
void pvfc(Flow& f) {
  const int n = f.n;
  for (size_t j = 0; j < f.w_cells.size(); ++j) f.pp[f.C(f.w_faces[j], f.w_cells[j])] = f.pp[f.w_cells[j]];
  grad_eval(f, f.gow, f.pp, f.dppx, f.dppy);
  for (int i = 1; i <= n; ++i) {
    if (f.iwet[i] == 0) continue;
    double val = f.h[i] * f.apuareap[i] / (1.0 - f.sumu[i] + 1.0e-15);
    f.u[i] = f.u[i] - val * f.dppx[i];
    f.v[i] = f.v[i] - val * f.dppy[i];
    for (int j = 1; j <= f.nxyface[i]; ++j) {
      int k = f.FI(f.kxyface, j, i), nck = f.C(k, i);
      if (f.iwet[nck] == 0) continue;
      f.F(f.flux, k, i) = f.F(f.flux, k, i) - f.F(f.acoef, k, i) * (f.pp[nck] - f.pp[i]);
      f.F(f.flux, f.FI(f.llec, k, i), nck) = -f.F(f.flux, k, i);
    }
  }
  if (f.skewcor) {
    for (int i : f.idjoint) {
      if (f.iwet[i] == 0) continue;
      for (int j = 1; j <= f.nxface[i]; ++j) {
        int k = f.FI(f.kxface, j, i), nck = f.C(k, i);
        if (nck > n || f.iwet[nck] == 0) continue;
        int jcn = f.FI(f.llec, k, i);
        if (std::fabs(f.F(f.rpy, k, i)) > 1.0e-6) {
          f.F(f.flux, k, i) = f.F(f.flux, k, i) + f.F(f.acoef, k, i) * f.F(f.rpy, k, i) * f.dppy[i];
          f.F(f.flux, jcn, nck) = -f.F(f.flux, k, i);
        } else if (std::fabs(f.F(f.rpy, jcn, nck)) > 1.0e-6) {
          f.F(f.flux, k, i) = f.F(f.flux, k, i) - f.F(f.acoef, k, i) * f.F(f.rpy, jcn, nck) * f.dppy[nck];
          f.F(f.flux, jcn, nck) = -f.F(f.flux, k, i);
        }
      }
      for (int j = 1; j <= f.nyface[i]; ++j) {
        int k = f.FI(f.kyface, j, i), nck = f.C(k, i);
        if (nck > n || f.iwet[nck] == 0) continue;
        int jcn = f.FI(f.llec, k, i);
        if (std::fabs(f.F(f.rpx, k, i)) > 1.0e-6) {
          f.F(f.flux, k, i) = f.F(f.flux, k, i) + f.F(f.acoef, k, i) * f.F(f.rpx, k, i) * f.dppx[i];
          f.F(f.flux, jcn, nck) = -f.F(f.flux, k, i);
        } else if (std::fabs(f.F(f.rpx, jcn, nck)) > 1.0e-6) {
          f.F(f.flux, k, i) = f.F(f.flux, k, i) - f.F(f.acoef, k, i) * f.F(f.rpx, jcn, nck) * f.dppx[nck];
          f.F(f.flux, jcn, nck) = -f.F(f.flux, k, i);
        }
      }
    }
  }
  const double gravinv = 1.0 / f.P.grav;
  for (int i = 1; i <= f.nD; ++i) {
    f.p[i] = f.p[i] + f.P.relax_p * f.pp[i];
    f.h[i] = std::max(f.P.hmin, f.p[i] * gravinv - f.zb[i]);
    f.pp[i] = f.P.facpp * f.pp[i];
  }
  for (size_t j = 0; j < f.w_cells.size(); ++j) f.p[f.C(f.w_faces[j], f.w_cells[j])] = f.p[f.w_cells[j]];
}

int solve(Flow& f, V& ss, V& sp, V& res, V& phi, int var, double* rmom_out) {
  // var: 1 pp, 2 u, 3 v.  Arrays are 1-based over ncellsD; the solver takes
  // 0-based rows, renumbered by perm when an ordering is set.
  const int nD = f.nD, nmf = f.nmf, n = f.n;
  const bool pm = !f.perm.empty();
  auto row_of = [&](int r) { return (pm && r < n) ? f.perm[r] : r; };  // solver row -> natural 0-based cell
  std::vector<double> a((size_t)nD * nmf), s0(nD), p0(nD), r0(nD), x0(nD);
  for (int r = 0; r < nD; ++r) {
    const int i = row_of(r) + 1;
    for (int k = 1; k <= nmf; ++k) a[(size_t)r * nmf + k - 1] = f.F(f.acoef, k, i);
    s0[r] = ss[i]; p0[r] = sp[i]; x0[r] = phi[i];
  }
  if (f.cap_var == var && !f.cap_done) {
    f.cap_acoef.assign((size_t)nD * nmf, 0.0);
    f.cap_ss.assign(nD, 0.0); f.cap_sp.assign(nD, 0.0); f.cap_phi.assign(nD, 0.0);
    for (int i = 1; i <= nD; ++i) {
      for (int k = 1; k <= nmf; ++k) f.cap_acoef[(size_t)(i - 1) * nmf + k - 1] = f.F(f.acoef, k, i);
      f.cap_ss[i - 1] = ss[i]; f.cap_sp[i - 1] = sp[i]; f.cap_phi[i - 1] = phi[i];
    }
    f.cap_done = 1;
  }
  double relax = var == 1 ? f.P.relax_pp : f.P.relax_uv;
  int nswp = var == 1 ? f.nswp_pp : f.nswp_uv;
  double rm = 0, rr = 0;
  int it = 0, inner = 0;
  int st;
  if (f.nsolv == 3 || f.nsolv == 4) {
    const int lfil = f.nsolv == 4 ? 8 : 35;
    st = orc_solve_d(pm ? f.solver_perm : f.solver, a.data(), s0.data(), p0.data(), r0.data(), x0.data(), relax,
                     nswp, f.nsolv, f.precond, f.tol, lfil, 1.0e-3, 0.5, &rm, &it, &inner, &rr, f.norm);
  } else {  // the other MATRIX_SOLVER options read the variable index (solvers.f90:242-289)
    st = orc_solve_n_d(pm ? f.solver_perm : f.solver, var, a.data(), s0.data(), p0.data(), r0.data(), x0.data(),
                       relax, nswp, f.nsolv, f.relaxsor, f.nswp_uv, f.precond, f.tol, &rm, &it, &inner, &rr,
                       f.norm);
  }
  f.solve_iters += it;
  for (int r = 0; r < nD; ++r) {
    const int i = row_of(r) + 1;
    ss[i] = s0[r]; res[i] = r0[r]; phi[i] = x0[r];
  }
  *rmom_out = rm;
  return st;
}

// check_conv (flow_imp.F90:1576-1747) with dtvar off
int check_conv(Flow& f, int niter, int maxit) {
  const Params& P = f.P;
  double* rmom = f.rmom;
  if (niter <= 2) {
    for (int q = 1; q <= 3; ++q) { f.rmom0[q] = std::max(rmom[q], 1e-15); f.rmom1[q] = f.rmom0[q]; }
  }
  double rmommax = std::max(rmom[1], std::max(rmom[2], rmom[3]));
  if (rmommax > 5.0) return 0;
  if (niter <= 5) return 1;
  int nhalf = maxit / 2;
  double rp = rmom[1] / f.rmom0[1];
  double ruv = std::max(rmom[2] / f.rmom0[2], rmom[3] / f.rmom0[3]);
  if ((rp >= P.rmomratiop * 10.0 || ruv >= P.rmomratiouv * 10.0) && rmom[1] > P.rmomtargetp) return 0;
  if (niter == maxit && (rp >= P.rmomratiop || ruv >= P.rmomratiouv) && rmom[1] > P.rmommaxp) return 0;
  if (niter == maxit && (rp >= P.rmomratiop / 5.0 || ruv >= P.rmomratiouv / 5.0) && rmom[1] > P.rmomtargetp)
    return P.dtvar ? 3 : 0;
  double rmomuv = std::max(rmom[2], rmom[3]);
  if (rmom[1] <= P.rmomminp && rmomuv <= P.rmomminuv) return 2;
  if (niter == maxit && (rmom[1] > P.rmommaxp || rmomuv > P.rmommaxuv)) return 0;
  if (niter == maxit && (rmom[1] > P.rmomtargetp || rmomuv > P.rmomtargetuv)) return P.dtvar ? 3 : 0;
  if (niter <= nhalf || niter % 2 != 0) return 1;
  double rchp = f.rmom1[1] - rmom[1];
  double rmomuv1 = std::max(f.rmom1[2], f.rmom1[3]);
  double rchuv = rmomuv1 - rmomuv;
  if (rchp < 0.0 || rchuv < 0.0) return 1;
  if (rchp <= P.rmomminp && rchuv <= P.rmomminuv) return 2;
  for (int q = 1; q <= 3; ++q) f.rmom1[q] = rmom[q];
  return 1;
}

// velface_eta (flow_imp.F90:1245-1573), Cartesian/telescoping branch
void velface_eta(Flow& f) {
  const double gravinv = 1.0 / f.P.grav;
  for (int i = 1; i <= f.n; ++i) {
    if (f.h[i] > f.P.hmin && f.iwet[i] == 1) {
      double umin = 1e6, umax = -1e6, vmin = 1e6, vmax = -1e6;
      for (int k = 1; k <= f.ncface[i]; ++k) {
        double vel = f.F(f.flux, k, i) / (f.F(f.hk, k, i) * f.F(f.ds, k, i));
        double uf = f.F(f.fnx, k, i) * vel, vf = f.F(f.fny, k, i) * vel;
        umin = std::min(umin, uf); umax = std::max(umax, uf);
        vmin = std::min(vmin, vf); vmax = std::max(vmax, vf);
      }
      f.u[i] = std::min(std::max(f.u[i], umin), umax);
      f.v[i] = std::min(std::max(f.v[i], vmin), vmax);
      f.eta[i] = f.p[i] * gravinv;
      f.uv[i] = std::sqrt(f.u[i] * f.u[i] + f.v[i] * f.v[i]);
    } else {
      f.h[i] = std::max(f.P.hmin, f.h[i]);
      f.u[i] = 0; f.v[i] = 0; f.uv[i] = 0; f.eta[i] = -999.0;
    }
  }
}

int flow_step(Flow& f, double dt, int maxit, int* niter_out) {
  // wetting and drying, then the gradient weights of changed cells (flow_imp.F90:73-79)
  flow_wetdry(f);
  f.last_nlist = der_update(f);
  solver_set_wet(f);
  srcsnk_static(f, dt);
  int iconv = 1, niter = 0;
  for (niter = 1; niter <= maxit; ++niter) {
    coef_uv(f);
    if (!f.idjoint.empty() && f.P.ndsch != 0) defcor(f);  // flow_imp.F90:127-138
    bound_uv(f);
    double rm = 0;
    int st = solve(f, f.su, f.spu, f.rsu, f.u, 2, &rm);
    f.rmom[2] = rm;
    if (st == 2) { iconv = 0; break; }
    st = solve(f, f.sv, f.spv, f.rsv, f.v, 3, &rm);
    f.rmom[3] = rm;
    if (st == 2) { iconv = 0; break; }
    coef_pp(f);
    bound_pp(f);
    st = solve(f, f.su, f.sp, f.rsp, f.pp, 1, &rm);
    f.rmom[1] = rm;
    if (st == 2) { iconv = 0; break; }
    pvfc(f);
    flow_grad_interp(f);
    fric_eval(f);
    flow_eddyvis(f);
    iconv = check_conv(f, niter, maxit);
    if (iconv == 0 || iconv == 2) break;
  }
  if (niter > maxit) niter = maxit;
  *niter_out = niter;
  f.last_niter = niter;
  f.last_iconv = iconv;
  velface_eta(f);
  fric_eval(f);
  // flow_update (CMS_Flow.f90:243-300), implicit branch
  for (int i = 1; i <= f.nD; ++i) {
    f.iwet1[i] = f.iwet[i];
    f.u1[i] = f.u[i]; f.v1[i] = f.v[i]; f.p1[i] = f.p[i]; f.h1[i] = f.h[i];
    f.pp[i] = 0.0; f.dppx[i] = 0.0; f.dppy[i] = 0.0;
  }
  return iconv == 0 ? 2 : 0;
}

}  // namespace

extern "C" {

// Creates the flow oracle: grid arrays 0-based C layout ([ncellsD][nmaxfaces]
// for cell2cell/idirface, 1-based neighbour ids), TH string (1-based cells and
// faces), coefman per cell, still water p = 0.
void* orcf_create(int ncells, int ncellsD, int nmf, const int* c2c, const int* ncface, const int* idirface,
                  const double* x, const double* y, const double* dx, const double* dy, const double* zb,
                  const double* coefman, int nth, const int* th_cells, const int* th_faces, int skewcor) {
  auto* f = new Flow();
  f->n = ncells; f->nD = ncellsD; f->nmf = nmf; f->NF = nmf + 1;
  const size_t FS = (size_t)(ncellsD + 1) * f->NF;
  f->c2c.assign(FS, 0); f->idir.assign(FS, 0); f->ncface.assign(ncellsD + 1, 0);
  for (V* a : {&f->x, &f->y, &f->dx, &f->dy, &f->zb}) a->assign(ncellsD + 1, 0.0);
  for (int i = 1; i <= ncellsD; ++i) {
    f->ncface[i] = ncface[i - 1];
    f->x[i] = x[i - 1]; f->y[i] = y[i - 1]; f->dx[i] = dx[i - 1]; f->dy[i] = dy[i - 1]; f->zb[i] = zb[i - 1];
    for (int k = 1; k <= nmf; ++k) {
      f->C(k, i) = c2c[(size_t)(i - 1) * nmf + k - 1];
      f->FI(f->idir, k, i) = idirface[(size_t)(i - 1) * nmf + k - 1];
    }
  }
  f->th_cells.assign(th_cells, th_cells + nth);
  f->th_faces.assign(th_faces, th_faces + nth);
  f->wsebnd.assign(nth, 0.0);
  // iwet: active wet; dummies of the TH string wet; all other dummies are walls (dry)
  f->iwet.assign(ncellsD + 1, 0);
  for (int i = 1; i <= ncells; ++i) f->iwet[i] = 1;
  std::vector<char> isth(FS, 0);
  for (int j = 0; j < nth; ++j) {
    isth[(size_t)th_cells[j] * f->NF + th_faces[j]] = 1;
    f->iwet[f->C(th_faces[j], th_cells[j])] = 1;
  }
  for (int i = 1; i <= ncells; ++i)
    for (int k = 1; k <= f->ncface[i]; ++k)
      if (f->C(k, i) > ncells && !isth[(size_t)i * f->NF + k]) { f->w_cells.push_back(i); f->w_faces.push_back(k); }
  f->skewcor = skewcor != 0;
  geometry(*f);
  if (f->idjoint.empty()) f->skewcor = false;  // flow.F90:832
  f->iwet1.assign(ncellsD + 1, 1);
  f->icorner.assign(ncellsD + 1, 0);
  for (int i = 1; i <= ncells; ++i) {
    int nd = 0;
    for (int k = 1; k <= f->ncface[i]; ++k) if (f->iwet[f->C(k, i)] == 0) ++nd;
    if (nd > 1) f->icorner[i] = 1;
  }
  build_go(*f, f->gow, 1);
  build_go(*f, f->goa, 0);
  for (V* a : {&f->p, &f->h, &f->u, &f->v, &f->pp, &f->eta, &f->vis, &f->cfrict, &f->uelwc, &f->uv, &f->bsxy,
               &f->bsvel, &f->z0, &f->coefman, &f->cmb, &f->fc, &f->u1, &f->v1, &f->p1, &f->h1, &f->su, &f->sv,
               &f->sp, &f->spu, &f->spv, &f->ssu0, &f->ssv0, &f->spuv0, &f->sppp0, &f->sspp0, &f->apuareap,
               &f->sumu, &f->Hu, &f->Hv, &f->cbcfuwcap, &f->dpx, &f->dpy, &f->dux, &f->duy, &f->dvx, &f->dvy,
               &f->dppx, &f->dppy, &f->dHux, &f->dHuy, &f->dHvx, &f->dHvy, &f->dapx, &f->dapy, &f->dzbx, &f->dzby,
               &f->rsu, &f->rsv, &f->rsp})
    a->assign(ncellsD + 1, 0.0);
  for (V* a : {&f->flux, &f->visk, &f->hk, &f->pk, &f->acoef, &f->zbk}) a->assign(FS, 0.0);
  for (int i = 1; i <= ncellsD; ++i) f->cmb[i] = 1.0;
  for (int i = 1; i <= ncells; ++i) f->coefman[i] = coefman[i - 1];
  std::vector<int> iw(ncellsD);
  for (int i = 1; i <= ncellsD; ++i) iw[i - 1] = f->iwet[i];
  f->solver = orc_create(ncells, ncellsD, nmf, c2c, ncface, iw.data(), 1);
  return f;
}

void orcf_destroy(void* h) {
  auto* f = static_cast<Flow*>(h);
  if (f->solver) orc_destroy(f->solver);
  if (f->solver_perm) orc_destroy(f->solver_perm);
  delete f;
}

// Solves the three systems in another unknown order: solver row r is natural
// cell perm[r] (0-based, ncells entries).  The ILU(0) factor then follows that
// order, as the GPU's multicolour or level order does.
void orcf_set_order(void* h, const int* perm) {
  auto* f = static_cast<Flow*>(h);
  const int n = f->n, nD = f->nD, nmf = f->nmf;
  f->perm.assign(perm, perm + n);
  f->iperm.assign(n, 0);
  for (int r = 0; r < n; ++r) f->iperm[perm[r]] = r;
  std::vector<int> c2c((size_t)nD * nmf, 0), ncf(nD), iw(nD);
  auto map = [&](int c) { return (c >= 1 && c <= n) ? f->iperm[c - 1] + 1 : c; };  // 1-based ids
  for (int r = 0; r < nD; ++r) {
    const int i = (r < n ? perm[r] : r) + 1;
    ncf[r] = f->ncface[i];
    iw[r] = f->iwet[i];
    for (int k = 1; k <= nmf; ++k) c2c[(size_t)r * nmf + k - 1] = map(f->C(k, i));
  }
  if (f->solver_perm) orc_destroy(f->solver_perm);
  f->solver_perm = orc_create(n, nD, nmf, c2c.data(), ncf.data(), iw.data(), 1);
}

void orcf_set_solver(void* h, int nsolv, int precond, double tol, int nswp_pp, int nswp_uv, int norm) {
  auto* f = static_cast<Flow*>(h);
  f->nsolv = nsolv; f->precond = precond; f->tol = tol; f->nswp_pp = nswp_pp; f->nswp_uv = nswp_uv; f->norm = norm;
}

// Cold start from the water level eta0 (ncellsD values) at rest (prestart.f90:
// 302-325): flow_wetdry(0) (again with ponding on when every cell is dry),
// iwet1 = iwet, and the wet-cell gradient operator of that wet set (der_init
// builds it from the wet set of flow_init's flow_wetdry call, which sees the
// same water level on a cold start).
int orcf_init(void* h, const double* eta0) {
  auto* f = static_cast<Flow*>(h);
  const double g = f->P.grav, gravinv = 1.0 / g;
  for (int i = 1; i <= f->nD; ++i) {
    f->p[i] = eta0[i - 1] * g;
    f->u[i] = f->v[i] = 0.0;
    f->iwet1[i] = 1;
  }
  flow_wetdry(*f);
  int nwet = 0;
  for (int i = 1; i <= f->n; ++i) nwet += f->iwet[i];
  if (nwet == 0) {
    f->P.ponding = true;
    flow_wetdry(*f);
  }
  for (int i = 1; i <= f->nD; ++i) {
    f->iwet1[i] = f->iwet[i];
    f->eta[i] = f->iwet[i] ? f->p[i] * gravinv : -999.0;
  }
  build_go(*f, f->gow, 1);
  solver_set_wet(*f);
  grad_eval(*f, f->goa, f->zb, f->dzbx, f->dzby);
  interp_c2f(*f, f->zb, 0, f->zbk, &f->dzbx, &f->dzby);
  flow_grad_interp(*f);
  std::fill(f->flux.begin(), f->flux.end(), 0.0);
  fric_eval(*f);
  flow_eddyvis(*f);
  for (int i = 1; i <= f->nD; ++i) { f->u1[i] = f->u[i]; f->v1[i] = f->v[i]; f->p1[i] = f->p[i]; f->h1[i] = f->h[i]; }
  return 0;
}

// flow_convflux (flow.F90:1879-1909): face fluxes from the cell velocities on
// each cell's no-repeat faces, copied with the opposite sign to the
// neighbour's face (bndflux adds nothing without flux or cross-shore strings).
void flow_convflux(Flow& f) {
  for (int i = 1; i <= f.n; ++i)
    for (int j = 1; j <= f.nxyface[i]; ++j) {
      const int k = f.FI(f.kxyface, j, i), nck = f.C(k, i), jcn = f.FI(f.llec, k, i);
      const double uni = f.F(f.fnx, k, i) * f.u[i] + f.F(f.fny, k, i) * f.v[i];
      const double unk = f.F(f.fnx, k, i) * f.u[nck] + f.F(f.fny, k, i) * f.v[nck];
      const double fk = f.F(f.fintp, k, i);
      f.F(f.flux, k, i) = (double)(f.iwet[i] * f.iwet[nck]) * f.F(f.ds, k, i) * f.F(f.hk, k, i) *
                          (fk * unk + (1.0 - fk) * uni);
      f.F(f.flux, jcn, nck) = -f.F(f.flux, k, i);
    }
}

// Hot start from the water pressure p and the velocities u, v of all ncellsD
// cells (what a hot-start file holds): hot_init (hot_start.F90:1125-1215) --
// h = p/g - zb; a cell with h < hmin + 1e-5 is dry (h = hmin, u = v = 0,
// eta = -999; p is kept, as when the file gave the pressure), else wet (eta =
// p/g); the dummy of each water-level string face takes its cell's u, v, p,
// eta and h; flow_update's time levels -- then the rest of prestart
// (prestart.f90:298-325): flow_wetdry(0) against hot_init's wet set (it wets
// cells with the dry-to-wet initialisation and zeroes the fluxes of dry
// faces), again with ponding on when every cell is dry; iwet1 = iwet; eta;
// bed slope and face beds; flow_grad_interp; flow_convflux unless the file
// held the face fluxes (flux != NULL, [ncellsD][nmaxfaces]); fric_eval;
// flow_eddyvis.  The wet-cell gradient operator is built from the wet set
// this start ends with (the reference builds it in der_init, before the hot
// start is read, from the wet set of the cold initial condition).
int orcf_init_hot(void* h, const double* p, const double* u, const double* v, const double* flux) {
  auto* f = static_cast<Flow*>(h);
  const double g = f->P.grav, gravinv = 1.0 / g;
  for (int i = 1; i <= f->nD; ++i) {
    f->p[i] = p[i - 1];
    f->u[i] = u[i - 1];
    f->v[i] = v[i - 1];
    f->vis[i] = 0.0;
    f->h[i] = f->p[i] * gravinv - f->zb[i];
    if (f->h[i] < f->P.hmin + 1.0e-5) {
      f->h[i] = f->P.hmin;
      f->iwet[i] = 0;
      f->u[i] = f->v[i] = 0.0;
      f->eta[i] = -999.0;
    } else {
      f->iwet[i] = 1;
      f->eta[i] = f->p[i] * gravinv;
    }
  }
  for (size_t j = 0; j < f->th_cells.size(); ++j) {
    const int i = f->th_cells[j], k = f->th_faces[j], nck = f->C(k, i);
    f->u[nck] = f->u[i]; f->v[nck] = f->v[i]; f->p[nck] = f->p[i]; f->eta[nck] = f->eta[i];
    f->zb[nck] = f->zb[i];
    f->h[i] = std::max(f->P.hmin, f->p[i] * gravinv - f->zb[i]);
    f->h[nck] = f->h[i];
  }
  for (int i = 1; i <= f->nD; ++i) f->iwet1[i] = f->iwet[i];
  std::fill(f->flux.begin(), f->flux.end(), 0.0);
  std::fill(f->visk.begin(), f->visk.end(), 0.0);
  if (flux)
    for (int i = 1; i <= f->nD; ++i)
      for (int k = 1; k <= f->nmf; ++k) f->F(f->flux, k, i) = flux[(size_t)(i - 1) * f->nmf + k - 1];
  flow_wetdry(*f);
  int nwet = 0;
  for (int i = 1; i <= f->n; ++i) nwet += f->iwet[i];
  if (nwet == 0) {
    f->P.ponding = true;
    flow_wetdry(*f);
  }
  for (int i = 1; i <= f->nD; ++i) {
    f->iwet1[i] = f->iwet[i];
    f->eta[i] = f->iwet[i] ? f->p[i] * gravinv : -999.0;
  }
  build_go(*f, f->gow, 1);
  solver_set_wet(*f);
  grad_eval(*f, f->goa, f->zb, f->dzbx, f->dzby);
  interp_c2f(*f, f->zb, 0, f->zbk, &f->dzbx, &f->dzby);
  flow_grad_interp(*f);
  if (!flux) flow_convflux(*f);
  fric_eval(*f);
  flow_eddyvis(*f);
  for (int i = 1; i <= f->nD; ++i) { f->u1[i] = f->u[i]; f->v1[i] = f->v[i]; f->p1[i] = f->p[i]; f->h1[i] = f->h[i]; }
  return 0;
}

// One implicit time step (flow_imp + flow_update).  wsebnd: water level of each
// TH-string cell.  Returns 0 ok, 2 divergent/non-finite.
int orcf_step(void* h, double dt, const double* wsebnd, int maxit, int* niter, double* rmom3) {
  auto* f = static_cast<Flow*>(h);
  for (size_t j = 0; j < f->wsebnd.size(); ++j) f->wsebnd[j] = wsebnd[j];
  int st = flow_step(*f, dt, maxit, niter);
  for (int q = 0; q < 3; ++q) rmom3[q] = f->rmom[q + 1];
  return st;
}

// Copies a state array: 0 p, 1 h, 2 u, 3 v, 4 eta, 5 vis, 6 cfrict, 7 dpx, 8 dpy
// (ncellsD values); 100 flux, 101 visk, 102 hk, 103 acoef, 104 fintp, 105 zbk
// ([ncellsD][nmaxfaces]); 200 iwet, 201 icorner (as values).  Returns the
// number of values.
long long orcf_get(void* h, int which, double* out) {
  auto* f = static_cast<Flow*>(h);
  if (which == 200 || which == 201) {
    const VI& a = which == 200 ? f->iwet : f->icorner;
    for (int i = 1; i <= f->nD; ++i) out[i - 1] = a[i];
    return f->nD;
  }
  if (which == 202) {  // cell area (geo_def areap)
    for (int i = 1; i <= f->nD; ++i) out[i - 1] = f->areap[i];
    return f->nD;
  }
  const V* cell[] = {&f->p, &f->h, &f->u, &f->v, &f->eta, &f->vis, &f->cfrict, &f->dpx, &f->dpy};
  const V* face[] = {&f->flux, &f->visk, &f->hk, &f->acoef, &f->fintp, &f->zbk, &f->dsxy};
  if (which >= 0 && which < 9) {
    for (int i = 1; i <= f->nD; ++i) out[i - 1] = (*cell[which])[i];
    return f->nD;
  }
  if (which >= 100 && which < 107) {
    const V& a = *face[which - 100];
    for (int i = 1; i <= f->nD; ++i)
      for (int k = 1; k <= f->nmf; ++k) out[(size_t)(i - 1) * f->nmf + k - 1] = a[(size_t)i * f->NF + k];
    return (long long)f->nD * f->nmf;
  }
  return -1;
}

long long orcf_solve_iters(void* h) { return static_cast<Flow*>(h)->solve_iters; }
// Arms the capture of the next solve() of variable var (1 pp, 2 u, 3 v).
void orcf_capture(void* h, int var) {
  Flow* f = static_cast<Flow*>(h);
  f->cap_var = var;
  f->cap_done = 0;
}
// The captured system (natural order, acoef [ncellsD][nmaxfaces]); 0 if none.
int orcf_captured(void* h, double* acoef, double* ss, double* sp, double* phi) {
  Flow* f = static_cast<Flow*>(h);
  if (!f->cap_done) return 0;
  std::copy(f->cap_acoef.begin(), f->cap_acoef.end(), acoef);
  std::copy(f->cap_ss.begin(), f->cap_ss.end(), ss);
  std::copy(f->cap_sp.begin(), f->cap_sp.end(), sp);
  std::copy(f->cap_phi.begin(), f->cap_phi.end(), phi);
  return 1;
}
// cells der_update recomputed at the start of the last step
int orcf_last_nlist(void* h) { return static_cast<Flow*>(h)->last_nlist; }
// ponding and narrowchannels switches (flow.F90:54-55)
void orcf_set_wetdry(void* h, int ponding, int narrowchannels) {
  auto* f = static_cast<Flow*>(h);
  f->P.ponding = ponding != 0;
  f->P.narrowchannels = narrowchannels != 0;
}
int orcf_njoint(void* h) { return (int)static_cast<Flow*>(h)->idjoint.size(); }
// ADVECTION_SCHEME card (flow.F90:533-545): 0 none .. 4 exponential
void orcf_set_scheme(void* h, int ndsch) { static_cast<Flow*>(h)->P.ndsch = ndsch; }
// DRYING_DEPTH card: hmin = hdry, hdry1 = 5 hdry, hdry2 = 2 hdry (flow.F90:686-693).
// The one- and two-cell depths only matter with narrow channels off, when
// flow.F90:686-689 overwrites the DRYING_DEPTH_ONE_CELL/TWO_CELL cards.
void orcf_set_hdry(void* h, double hdry) {
  auto* f = static_cast<Flow*>(h);
  f->P.hmin = hdry; f->P.hdry = hdry; f->P.hdry1 = 5.0 * hdry; f->P.hdry2 = 2.0 * hdry;
}

}  // extern "C"
