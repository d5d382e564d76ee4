// Device kernels of the implicit flow step (SIMPLEC outer iteration).
//
// Layout.  Cells are numbered in the solver's device order: active cells
// 0..n-1 (colour groups, natural order inside a group), then the dummy cells
// n..nD-1 in their natural order.  Face arrays are slot-major,
// A[k * nD + r] for face k (0..nmf-1) of cell r, so a warp reading face k of
// 32 consecutive cells touches one contiguous segment.  A face shared by two
// cells is evaluated once by the cell that owns it (the reference's no-repeat
// face lists) and mirrored into the neighbour's slot, as the reference does.
#pragma once
#include "cms_common.cuh"

namespace cms {

struct FlowDev {
  int n, nD, nmf, nsc, ider;
  int ndsch;  // advection scheme of the momentum coefficients (0 none, 1 upwind, 2 hybrid, 3 power law, 4 exponential)
  // connectivity (device numbering)
  const int* ncface;          // [nD]
  const int* nb;              // [nmf][nD] neighbour (dummies >= n), -1 none
  const signed char* back;    // [nmf][nD] face index seen from the neighbour
  const signed char* dir;     // [nmf][nD] 1..4 = N,E,S,W
  const unsigned char* owned; // [nD] bit k: face k is on the cell's no-repeat list
  const unsigned char* thm;   // [nD] bit k: face k is on a water-level string
  const unsigned char* joint; // [nD]
  const unsigned char* crmask;  // [nD] bit k: face k takes part in the cell-reconstruction weights
  const int* iwet;            // [nD]
  // metrics
  const double *ds, *dn, *dsxy, *rx, *ry, *rpx, *rpy, *fintp;  // [nmf][nD]
  const double *areap, *zb, *coefman;                          // [nD]
  // gradient operator (wet cells): [q][n] stencils
  const int *ncx, *ncy, *icx, *icy, *ngx, *ngy, *igx, *igy;
  const double *wcx, *wcy, *wgxy, *wgyx;
  // parameters
  double grav, gravinv, hmin, hdry, hdry1, hdry2, relax_uv, relax_p, facpp, cviscon, cvisbot, cvishor2areaavg,
      cvismax, wallfac;
};

// The wet-cell gradient operator as written by kf_gw_rows (the same buffers
// FlowDev reads).
struct GWOut {
  int *ncx, *ncy, *icx, *icy, *ngx, *ngy, *igx, *igy;
  double *wcx, *wcy, *wgxy, *wgyx;
};

__device__ __forceinline__ int fidx(const FlowDev& G, int k, int r) { return k * G.nD + r; }
__device__ __forceinline__ double fnxd(int d) { return d == 2 ? 1.0 : (d == 4 ? -1.0 : 0.0); }
__device__ __forceinline__ double fnyd(int d) { return d == 1 ? 1.0 : (d == 3 ? -1.0 : 0.0); }

__device__ __forceinline__ double expcoef(double dk, double fk) {  // comp_lib.f90:96-109
  const double absfk = fabs(fk);
  const double peck = absfk / fmax(fmax(dk, 1.0e-6), absfk);
  return dk * peck / fmax(exp(peck) - 1.0, 1.0e-6) + fmax(0.0, -fk);
}
__device__ __forceinline__ double upwcoef(double dk, double fk) { return dk + fmax(0.0, -fk); }  // comp_lib.f90:54-64
__device__ __forceinline__ double hybcoef(double dk, double fk) {  // comp_lib.f90:67-78
  const double peck = fabs(fk) / fmax(dk, 1.0e-6);
  return dk * fmax(0.0, 1.0 - 0.5 * peck) + fmax(0.0, -fk);
}
__device__ __forceinline__ double powcoef(double dk, double fk) {  // comp_lib.f90:81-93
  const double absfk = fabs(fk);
  const double peck = absfk / fmax(fmax(dk, absfk), 1.0e-6);
  const double p2 = peck * peck;
  return dk * (1.0 - p2 * p2 * peck) + fmax(0.0, -fk);
}
// the momentum face coefficient of the selected scheme (the coefficient
// function coeffsourcesink_uv is called with, flow_imp.F90:120-126)
__device__ __forceinline__ double schemecoef(int ndsch, double dk, double fk) {
  switch (ndsch) {
    case 0: return 0.0;  // zerocoef, comp_lib.f90:40-51
    case 2: return hybcoef(dk, fk);
    case 3: return powcoef(dk, fk);
    case 4: return expcoef(dk, fk);
    default: return upwcoef(dk, fk);
  }
}
__device__ __forceinline__ double wallcoef(double yp, double y0) {  // fric_lib.f90:162-194
  const double y0lim = fmin(fmax(y0, 1.0e-6), yp * 0.9999);
  const double c = 0.4 / log(yp / y0lim);
  return c * c;
}

struct FlowState {
  double *p, *h, *u, *v, *pp, *vis, *vis0, *vis1, *cfrict, *z0, *uv, *bsvel, *eta;
  double *u1, *v1, *p1, *h1;
  double *su, *sv, *sp, *spu, *spv, *ssu0, *ssv0, *spuv0, *sppp0, *sspp0, *apuareap, *sumu, *Hu, *Hv, *res;
  double *flux, *visk, *hk, *pk, *acoef, *zbk;  // faces
  // gradients, two copies each (the cell-reconstruction correction reads the previous one)
  double *dpx[2], *dpy[2], *dux[2], *duy[2], *dvx[2], *dvy[2], *dppx[2], *dppy[2];
  double *dHux[2], *dHuy[2], *dHvx[2], *dHvy[2], *dapx[2], *dapy[2], *dzbx[2], *dzby[2];
  double* wsebnd;      // [nth]
  int* flag;           // [4] device status flags: 1 non-finite, 2 depth classes changed, 3 cells in chg
  int* chg;            // [nD] cells whose depth classes changed: row | classes << 28
};

// depth h = p/g - zb with two roundings (as the host and the reference form it)
__device__ __forceinline__ double depth_of(const FlowDev& G, double p, double zb) {
  return __dsub_rn(__dmul_rn(p, G.gravinv), zb);
}

// ----------------------------------------------------------------------------
// flow_srcsnk_static, ntsch = 1 (flow_imp.F90:336-346), plus the depth update of
// flow_wetdry(0) (flow.F90:1247-1255).
__global__ void __launch_bounds__(TPB) kf_static(FlowDev G, FlowState S, double dt) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.nD) return;
  double hh = depth_of(G, S.p[r], G.zb[r]);
  if (hh < G.hdry) hh = fmax(hh, G.hmin);
  S.h[r] = hh;
  if (r >= G.n) return;
  const double fac1 = G.areap[r] * S.h1[r] / dt;
  S.spuv0[r] = -fac1;
  S.ssu0[r] = fac1 * S.u1[r];
  S.ssv0[r] = fac1 * S.v1[r];
  S.sppp0[r] = -G.areap[r] / (G.grav * dt);
  S.sspp0[r] = -S.p1[r] * S.sppp0[r];
}

// skew term of face k of joint cell r, owner-side formula of defcorparagradvec
// (computational.F90:175-213) evaluated for (owner o, its face ko).
__device__ __forceinline__ void defcor_face(const FlowDev& G, const FlowState& S, int o, int ko, const double* dux,
                                            const double* duy, const double* dvx, const double* dvy, double& us,
                                            double& vs) {
  us = 0.0; vs = 0.0;
  const int f = fidx(G, ko, o);
  const int nck = G.nb[f];
  if (G.iwet[o] == 0 || nck >= G.n || G.iwet[nck] == 0) return;
  const int jcn = G.back[f];
  const int fb = fidx(G, jcn, nck);
  const int d = G.dir[f];
  const bool xface = (d == 2 || d == 4);
  const double rpk = xface ? G.rpy[f] : G.rpx[f];
  const double rpn = xface ? G.rpy[fb] : G.rpx[fb];
  // acoef of the face from its own inputs (the momentum coefficient of (ko, o))
  const double a = schemecoef(G.ndsch, S.visk[f] * S.hk[f] * G.dsxy[f], S.flux[f]);
  if (fabs(rpk) > 1.0e-6) {
    const double val = (a + S.flux[f]) * rpk;
    us = val * (xface ? duy[o] : dux[o]);
    vs = val * (xface ? dvy[o] : dvx[o]);
  } else if (fabs(rpn) > 1.0e-6) {
    const double val = -a * rpn;
    us = val * (xface ? duy[nck] : dux[nck]);
    vs = val * (xface ? dvy[nck] : dvx[nck]);
  }
}

// coeffsourcesink_uv(schemecoef) (flow_imp.F90:409-466), the skewness
// deferred correction of joint cells (defcorparagradvec), and bound_uv
// (boundaries.F90:3310-3490): water-level string faces (bnd_vel_openwse,
// bnd_vel.f90:35-95) then wall friction (wallfric) or dry-cell rows.
__global__ void __launch_bounds__(TPB) kf_coef_uv(FlowDev G, FlowState S, const double* dux, const double* duy,
                                                  const double* dvx, const double* dvy, const double* dpx,
                                                  const double* dpy) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  const double h = S.h[r], A = G.areap[r];
  const double fc = 0.0;  // Coriolis parameter (fcoriolis = 0, flow.F90:60)
  double su = S.ssu0[r] + (fc * S.v[r] - dpx[r]) * h * A;
  double sv = S.ssv0[r] + (-fc * S.u[r] - dpy[r]) * h * A;
  const double cb = 1.0 * S.cfrict[r] * S.uv[r] * A;
  double sp = S.spuv0[r] - cb;
  const int nf = G.ncface[r];
  for (int k = 0; k < nf; ++k) {
    const int f = fidx(G, k, r);
    S.acoef[f] = schemecoef(G.ndsch, S.visk[f] * S.hk[f] * G.dsxy[f], S.flux[f]);
  }
  // deferred skewness correction of joint cells: every first-order scheme
  // but NONE (flow_imp.F90:127-138)
  if (G.ider == 2 && G.joint[r] && G.ndsch != 0) {
    double ssu = 0.0, ssv = 0.0;
    for (int k = 0; k < nf; ++k) {
      double us = 0.0, vs = 0.0;
      if ((G.owned[r] >> k) & 1) {
        defcor_face(G, S, r, k, dux, duy, dvx, dvy, us, vs);
      } else {
        const int nck = G.nb[fidx(G, k, r)];
        if (nck < G.n && G.joint[nck]) {
          defcor_face(G, S, nck, G.back[fidx(G, k, r)], dux, duy, dvx, dvy, us, vs);
          us = -us; vs = -vs;
        }
      }
      ssu = ssu + us;
      ssv = ssv + vs;
    }
    su = su - ssu;
    sv = sv - ssv;
  }
  // water-level string faces
  const unsigned char tm = G.thm[r];
  if (tm) {
    for (int k = 0; k < nf; ++k) {
      if (!((tm >> k) & 1)) continue;
      const int f = fidx(G, k, r);
      const int nck = G.nb[f];
      const double a = upwcoef(S.visk[f] * S.hk[f] * G.dsxy[f], S.flux[f]);
      const int d = G.dir[f];
      if (d == 1 || d == 3) {
        S.u[nck] = G.iwet[r] * S.u[r] * h / S.h[nck];
        const double vg = fnyd(d) * S.flux[f] / (G.ds[f] * S.hk[f]);
        S.v[nck] = vg;
        sv = sv + a * vg;
      } else {
        const double ug = fnxd(d) * S.flux[f] / (G.ds[f] * S.hk[f]);
        S.u[nck] = ug;
        S.v[nck] = G.iwet[r] * S.v[r] * h / S.h[nck];
        su = su + a * ug;
      }
      sp = sp - a;
      S.acoef[f] = 0.0;
    }
  }
  double spu = sp, spv = sp;
  if (G.iwet[r] == 1) {
    for (int k = 0; k < nf; ++k) {
      const int f = fidx(G, k, r);
      const int nck = G.nb[f];
      if (G.iwet[nck] != 0) continue;
      const double z0w = S.z0[r] * G.wallfac;
      const int d = G.dir[f];
      if (d == 1 || d == 3) {
        spu = spu - G.ds[f] * S.hk[f] * wallcoef(fabs(G.ry[f]), z0w) * fabs(S.u[r]);
      } else {
        spv = spv - G.ds[f] * S.hk[f] * wallcoef(fabs(G.rx[f]), z0w) * fabs(S.v[r]);
      }
    }
  } else {
    S.u[r] = 0.0; S.v[r] = 0.0;
    spu = -1.0; spv = -1.0; sp = -1.0;
    su = 0.0; sv = 0.0;
  }
  S.su[r] = su; S.sv[r] = sv; S.sp[r] = sp; S.spu[r] = spu; S.spv[r] = spv;
}

// coefsourcesink_pp, cell part (flow_imp.F90:604-617)
__global__ void __launch_bounds__(TPB) kf_pp_cell(FlowDev G, FlowState S, const double* dpx, const double* dpy) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  double asum = 0.0;
  const int nf = G.ncface[r];
  for (int k = 0; k < nf; ++k) asum = asum + S.acoef[fidx(G, k, r)];
  const double apu = G.iwet[r] * G.relax_uv / fmax(asum - S.sp[r], 1.0e-6);
  const double ap = apu * G.areap[r];
  S.apuareap[r] = ap;
  S.sumu[r] = asum * apu;
  S.Hu[r] = G.iwet[r] * (S.u[r] + ap * dpx[r] * S.h[r]);
  S.Hv[r] = G.iwet[r] * (S.v[r] + ap * dpy[r] * S.h[r]);
}

// Cell-based Green-Gauss gradient of one or two scalars (der_grad_eval,
// der_lib.f90:726-842; der_gradvec_eval 936-1049) with the lagged
// cell-reconstruction correction of joint cells (reads the previous gradient).
template <int NV>
__global__ void __launch_bounds__(TPB) kf_grad(FlowDev G, const double* a, const double* b, double* ax, double* ay,
                                               double* bx, double* by, const double* axm, const double* aym,
                                               const double* bxm, const double* bym) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  double gax = 0.0, gbx = 0.0, gay = 0.0, gby = 0.0;
  const int nx = G.ncx[r], ny = G.ncy[r];
  for (int q = 0; q < nx; ++q) {
    const int c = G.icx[q * G.n + r];
    const double w = G.wcx[q * G.n + r];
    gax = gax + w * a[c];
    if (NV == 2) gbx = gbx + w * b[c];
  }
  for (int q = 0; q < ny; ++q) {
    const int c = G.icy[q * G.n + r];
    const double w = G.wcy[q * G.n + r];
    gay = gay + w * a[c];
    if (NV == 2) gby = gby + w * b[c];
  }
  if (G.ider == 2 && G.joint[r]) {
    const int mx = G.ngx[r], my = G.ngy[r];
    for (int q = 0; q < mx; ++q) {
      const int c = G.igx[q * G.n + r];
      const double w = G.wgxy[q * G.n + r];
      gax = gax + w * aym[c];
      if (NV == 2) gbx = gbx + w * bym[c];
    }
    for (int q = 0; q < my; ++q) {
      const int c = G.igy[q * G.n + r];
      const double w = G.wgyx[q * G.n + r];
      gay = gay + w * axm[c];
      if (NV == 2) gby = gby + w * bxm[c];
    }
  }
  ax[r] = gax; ay[r] = gay;
  if (NV == 2) { bx[r] = gbx; by[r] = gby; }
}

// Pressure-correction coefficients on owned faces, mirrored (flow_imp.F90:
// 622-649), and the Rhie-Chow face flux (flow_imp_flux_skew, flow_imp_flux.f90:
// 2-169, or _noskew 361-409).
__global__ void __launch_bounds__(TPB) kf_pp_face(FlowDev G, FlowState S, int skew, const double* dHuy,
                                                  const double* dHvx, const double* dapx, const double* dapy,
                                                  const double* dpx, const double* dpy) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  const unsigned char own = G.owned[r];
  const int nf = G.ncface[r];
  const bool jr = skew && G.joint[r];
  for (int k = 0; k < nf; ++k) {
    if (!((own >> k) & 1)) continue;
    const int f = fidx(G, k, r);
    const int nck = G.nb[f];
    const int fb = fidx(G, G.back[f], nck);
    const double hk = S.hk[f], ds = G.ds[f], dn = G.dn[f];
    double a, fl;
    const int d = G.dir[f];
    const double fnx = fnxd(d), fny = fnyd(d);
    if (G.iwet[r] * G.iwet[nck] == 0) {
      a = 0.0;
      fl = 0.0;
    } else if (nck >= G.n) {
      a = hk * hk * ds * S.apuareap[r] / (1.0 - S.sumu[r]) / dn;
      if (skew) {
        const bool xface = (d == 2 || d == 4);
        fl = hk * ds * ((xface ? fnx * S.Hu[r] : fny * S.Hv[r]) - S.apuareap[r] * hk * (S.p[nck] - S.p[r]) / dn);
      } else {
        fl = hk * ds * ((fnx * S.Hu[r] + fny * S.Hv[r]) - S.apuareap[r] * hk * (S.p[nck] - S.p[r]) / dn);
      }
    } else {
      const double fk = G.fintp[f], fp = 1.0 - fk;
      const double apv = fk * S.apuareap[nck] + fp * S.apuareap[r];
      const double suf = fk * S.sumu[nck] + fp * S.sumu[r];
      a = hk * hk * ds * apv / (1.0 - suf) / dn;
      if (!skew) {
        const double huf = fk * S.Hu[nck] + fp * S.Hu[r], hvf = fk * S.Hv[nck] + fp * S.Hv[r];
        fl = hk * ds * ((fnx * huf + fny * hvf) - apv * hk * (S.p[nck] - S.p[r]) / dn);
      } else {
        const bool xface = (d == 2 || d == 4);
        const double fn = xface ? fnx : fny;
        const double* H = xface ? S.Hu : S.Hv;
        if (!jr) {
          const double hf = fk * H[nck] + fp * H[r];
          fl = hk * ds * (fn * hf - apv * hk * (S.p[nck] - S.p[r]) / dn);
        } else {
          const double rpk = xface ? G.rpy[f] : G.rpx[f];
          const double rpn = xface ? G.rpy[fb] : G.rpx[fb];
          const double* dap = xface ? dapy : dapx;
          const double* dH = xface ? dHuy : dHvx;
          const double* dp = xface ? dpy : dpx;
          double ap2, hf, dpf;
          if (fabs(rpk) > 1.0e-6) {
            ap2 = fk * S.apuareap[nck] + fp * (S.apuareap[r] + rpk * dap[r]);
            hf = fk * H[nck] + fp * (H[r] + rpk * dH[r]);
            dpf = (S.p[nck] - S.p[r] - rpk * dp[r]) / dn;
          } else if (fabs(rpn) > 1.0e-6) {
            ap2 = fk * (S.apuareap[nck] + rpn * dap[nck]) + fp * S.apuareap[r];
            hf = fk * (H[nck] + rpn * dH[nck]) + fp * H[r];
            dpf = (S.p[nck] + rpn * dp[nck] - S.p[r]) / dn;
          } else {
            ap2 = apv;
            hf = fk * H[nck] + fp * H[r];
            dpf = (S.p[nck] - S.p[r]) / dn;
          }
          fl = hk * ds * (fn * hf - ap2 * hk * dpf);
        }
      }
    }
    S.acoef[f] = a;
    S.acoef[fb] = a;
    S.flux[f] = fl;
    S.flux[fb] = -fl;
  }
}

// skew term fcorr of face (ko, o) for the pressure-correction source
// (flow_imp.F90:720-765), owner side
__device__ __forceinline__ double fcorr_face(const FlowDev& G, const FlowState& S, int o, int ko, const double* dppx,
                                             const double* dppy) {
  const int f = fidx(G, ko, o);
  const int nck = G.nb[f];
  if (G.iwet[o] == 0 || G.iwet[nck] == 0) return 0.0;
  const int fb = fidx(G, G.back[f], nck);
  const int d = G.dir[f];
  const bool xface = (d == 2 || d == 4);
  const double rpk = xface ? G.rpy[f] : G.rpx[f];
  const double rpn = (nck < G.nD) ? (xface ? G.rpy[fb] : G.rpx[fb]) : 0.0;
  const double* dpp = xface ? dppy : dppx;
  if (fabs(rpk) > 1.0e-6) return -S.acoef[f] * rpk * dpp[o];
  if (fabs(rpn) > 1.0e-6) return S.acoef[f] * rpn * dpp[nck];
  return 0.0;
}

// Pressure-correction source terms (flow_imp.F90:699-711, skew 713-789) and
// bound_pp for water-level strings (bnd_pp, boundaries.F90:4767-4795) and dry
// rows (3493-3537).
__global__ void __launch_bounds__(TPB) kf_pp_src(FlowDev G, FlowState S, int skew, const double* dppx,
                                                 const double* dppy, const double* wse_of_cell) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  const int nf = G.ncface[r];
  double sp = S.sppp0[r];
  double sf = 0.0;
  for (int k = 0; k < nf; ++k) sf = sf + S.flux[fidx(G, k, r)];
  double su = S.sspp0[r] - sf + S.p[r] * sp;
  if (skew && G.joint[r]) {
    double fc = 0.0;
    for (int k = 0; k < nf; ++k) {
      double v = 0.0;
      if ((G.owned[r] >> k) & 1) {
        v = fcorr_face(G, S, r, k, dppx, dppy);
      } else {
        const int nck = G.nb[fidx(G, k, r)];
        if (nck < G.n && G.joint[nck]) v = -fcorr_face(G, S, nck, G.back[fidx(G, k, r)], dppx, dppy);
      }
      fc = fc + v;
    }
    su = su + 0.2 * fc;
  }
  if (G.iwet[r] == 0) {
    int sumwet = 0;
    for (int k = 0; k < nf; ++k) { const int c = G.nb[fidx(G, k, r)]; if (c < G.n) sumwet += G.iwet[c]; }
    double aploc = 0.0;
    su = 0.0;
    for (int k = 0; k < nf; ++k) {
      const int f = fidx(G, k, r), c = G.nb[f];
      double a;
      if (sumwet >= 1) a = G.iwet[c];
      else if (c >= G.n) { S.acoef[f] = 0.0; continue; }
      else a = G.dsxy[f];
      S.acoef[f] = a;
      aploc = aploc + a;
      su = su + a * S.p[c];
    }
    su = su - aploc * S.p[r];
    sp = 0.0;
  }
  const unsigned char tm = G.thm[r];
  if (tm) {
    for (int k = 0; k < nf; ++k) {
      if (!((tm >> k) & 1)) continue;
      const int f = fidx(G, k, r), c = G.nb[f];
      const double ppg = wse_of_cell[c] * G.grav - S.p[c];
      S.pp[c] = ppg;
      su = su + S.acoef[f] * ppg;
      sp = sp - S.acoef[f];
      S.acoef[f] = 0.0;
    }
  }
  S.su[r] = su;
  S.sp[r] = sp;
}

// pvfc (flow_imp.F90:797-1072), part 1: wall dummies take pp of their cell.
__global__ void kf_wall_copy(const int* wc, const int* wg, int nw, double* a) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j < nw) a[wg[j]] = a[wc[j]];
}

// pvfc part 2: velocity and flux corrections (owned faces, mirrored), skew
// corrections of joint cells' flux.
__global__ void __launch_bounds__(TPB) kf_pvfc(FlowDev G, FlowState S, int skew, const double* dppx,
                                               const double* dppy) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n || G.iwet[r] == 0) return;
  const double val = S.h[r] * S.apuareap[r] / (1.0 - S.sumu[r] + 1.0e-15);
  S.u[r] = S.u[r] - val * dppx[r];
  S.v[r] = S.v[r] - val * dppy[r];
  const unsigned char own = G.owned[r];
  const int nf = G.ncface[r];
  const bool jr = skew && G.joint[r];
  for (int k = 0; k < nf; ++k) {
    if (!((own >> k) & 1)) continue;
    const int f = fidx(G, k, r), nck = G.nb[f];
    if (G.iwet[nck] == 0) continue;
    const int fb = fidx(G, G.back[f], nck);
    double fl = S.flux[f] - S.acoef[f] * (S.pp[nck] - S.pp[r]);
    if (jr && nck < G.n) {
      const int d = G.dir[f];
      const bool xface = (d == 2 || d == 4);
      const double rpk = xface ? G.rpy[f] : G.rpx[f];
      const double rpn = xface ? G.rpy[fb] : G.rpx[fb];
      const double* dpp = xface ? dppy : dppx;
      if (fabs(rpk) > 1.0e-6) fl = fl + S.acoef[f] * rpk * dpp[r];
      else if (fabs(rpn) > 1.0e-6) fl = fl - S.acoef[f] * rpn * dpp[nck];
    }
    S.flux[f] = fl;
    S.flux[fb] = -fl;
  }
}

// pvfc part 3: p += relax*pp; h = max(hmin, p/g - zb); pp *= facpp (all cells)
__global__ void __launch_bounds__(TPB) kf_pvfc_p(FlowDev G, FlowState S) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.nD) return;
  const double p = S.p[r] + G.relax_p * S.pp[r];
  S.p[r] = p;
  S.h[r] = fmax(G.hmin, p * G.gravinv - G.zb[r]);
  S.pp[r] = G.facpp * S.pp[r];
}

// interp_scal_cell2face (interp_lib.f90:2727-2906) on owned faces, mirrored:
// ibc 0 (no treatment), 1 (zero gradient at wet/dry faces) or 3 (zero at dry
// faces), with the skewness correction of joint cells when dphix is given.
__global__ void __launch_bounds__(TPB) kf_interp(FlowDev G, const double* phi, int ibc, double* phik,
                                                 const double* dphix, const double* dphiy) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  const unsigned char own = G.owned[r];
  const int nf = G.ncface[r];
  const bool corr = dphix != nullptr && G.joint[r];
  for (int k = 0; k < nf; ++k) {
    if (!((own >> k) & 1)) continue;
    const int f = fidx(G, k, r), nck = G.nb[f];
    const int fb = fidx(G, G.back[f], nck);
    const double fk = G.fintp[f];
    const int wr = G.iwet[r], wn = G.iwet[nck];
    double v;
    if (ibc == 0) v = fk * phi[nck] + (1.0 - fk) * phi[r];
    else if (ibc == 1) {
      if (wr * wn == 1) v = fk * phi[nck] + (1.0 - fk) * phi[r];
      else if (wr == 1) v = phi[r];
      else if (wn == 1) v = phi[nck];
      else v = 0.5 * (phi[r] + phi[nck]);
    } else {
      v = (wr * wn == 1) ? fk * phi[nck] + (1.0 - fk) * phi[r] : 0.0;
    }
    if (corr) {
      const int d = G.dir[f];
      if (d == 2 || d == 4)
        v = v + fk * G.rpy[fb] * dphiy[nck] + (1.0 - fk) * G.rpy[f] * dphiy[r];
      else
        v = v + fk * G.rpx[fb] * dphix[nck] + (1.0 - fk) * G.rpx[f] * dphix[r];
      v = fmin(fmax(v, fmin(phi[r], phi[nck])), fmax(phi[r], phi[nck]));
    }
    phik[f] = v;
    phik[fb] = v;
  }
}

// flow_grad_interp, cell part (flow_imp.F90:1117-1127): dpx, dpy from face
// pressures and the face depths hk.
__global__ void __launch_bounds__(TPB) kf_dp_hk(FlowDev G, FlowState S, double* dpx, double* dpy) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  double ax = 0.0, ay = 0.0;
  const int nf = G.ncface[r];
  for (int k = 0; k < nf; ++k) {
    const int f = fidx(G, k, r);
    const int d = G.dir[f];
    const double pk = S.pk[f];
    ax = ax + fnxd(d) * G.ds[f] * pk;
    ay = ay + fnyd(d) * G.ds[f] * pk;
    S.hk[f] = fmax(G.hmin, pk * G.gravinv - S.zbk[f]);
  }
  dpx[r] = ax / G.areap[r];
  dpy[r] = ay / G.areap[r];
}

// fric_eval: Manning (friction.F90:647-662, fric_lib.f90:944-996) and
// fric_curmean_quad (877-905); the eddy viscosity of wet cells, mturbul = 5
// (flow_eddyvis.f90:136-146).
__global__ void __launch_bounds__(TPB) kf_fric_vis(FlowDev G, FlowState S, const double* dux, const double* duy,
                                                   const double* dvx, const double* dvy, int do_vis) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  const double h = S.h[r];
  const double cman = G.coefman[r];
  const double hh = fmax(fmin(10.0, h), 0.1 * cman);
  const double cd = G.grav * cman * cman / pow(hh, 0.3333);
  S.cfrict[r] = cd;
  if (cd != 0.0) S.z0[r] = fmax(h / exp(0.4 / sqrt(cd) + 1.0), 1.0e-6);
  const double um = sqrt(S.u[r] * S.u[r] + S.v[r] * S.v[r]);
  S.uv[r] = um;
  const double taum = 1025.0 * cd * um * um;
  const double bsv = sqrt(taum / 1025.0 + 1.0e-15);
  S.bsvel[r] = bsv;
  if (!do_vis) return;
  double vis;
  if (G.iwet[r] == 1) {
    const double a = dux[r], b = dvy[r], c = duy[r] + dvx[r];
    const double st = sqrt(2.0 * (a * a + b * b) + c * c);
    vis = fmin(G.cviscon + G.cvisbot * bsv * h + G.cvishor2areaavg * st, G.cvismax);
  } else {
    vis = 1.0e-6;
  }
  S.vis[r] = vis;
}

// eddy viscosity next to dry/dummy neighbours (flow_eddyvis.f90:169-186),
// run level by level so that the natural-order recurrence is reproduced.
// Each wall face of list cell r (a face to a dry cell or a dummy) sets
// vis(r) and vis of that neighbour from r's cells on the opposite side.
// Reads: an earlier list cell (rd_cur bit kk) is read updated, a later or
// unlisted wet cell as it was before this pass (vis0); r's own dummy as it
// is in memory (only r writes it); a dry active cell as the last write to it
// in cell order: r's own write at an earlier face kk < k, else the face value
// of the last earlier list cell that wrote it (src[j*nmf+kk], a face index
// into wallv; -1: before this pass).  Several list cells can write one dry
// cell, so those writes go to the face array wallv and kf_vis_wall_final
// copies the last writer's value in.
__global__ void kf_vis_wall(FlowDev G, FlowState S, const int* cells, const unsigned char* rd_cur, const int* src,
                            double* wallv, int m) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j >= m) return;
  const int r = cells[j];
  const unsigned char cur = rd_cur[j];
  const int nf = G.ncface[r];
  static constexpr int kk_of[5] = {0, 3, 4, 1, 2};
  for (int k = 0; k < nf; ++k) {
    const int f = fidx(G, k, r), nck = G.nb[f];
    if (!(G.iwet[nck] == 0 || nck >= G.n)) continue;
    const int kkdf = kk_of[G.dir[f]];
    double cid = 0.0, vs = 0.0;
    for (int kk = 0; kk < nf; ++kk) {
      const int fk = fidx(G, kk, r);
      if (G.dir[fk] != kkdf) continue;
      const int c = G.nb[fk];
      double vc;
      if (c >= G.n) {
        vc = S.vis[c];
      } else if (G.iwet[c] == 0) {
        const int sf = src[j * G.nmf + kk];
        vc = kk < k ? wallv[fk] : (sf >= 0 ? wallv[sf] : S.vis0[c]);
      } else {
        vc = ((cur >> kk) & 1) ? S.vis[c] : S.vis0[c];
      }
      cid = cid + 1.0;
      vs = vs + vc - G.cviscon;
    }
    const double vi = G.cviscon + vs / (cid + 1.0e-15);
    S.vis[r] = vi;
    if (nck >= G.n) S.vis[nck] = vi;
    else wallv[f] = vi;
  }
}

// dry active cells written by the wall pass take their last writer's value
__global__ void kf_vis_wall_final(const int* cells, const int* faces, int m, const double* wallv, double* vis) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j < m) vis[cells[j]] = wallv[faces[j]];
}

// corner cells (flow_eddyvis.f90:199-209), level by level like kf_vis_wall
__global__ void kf_vis_corner(FlowDev G, FlowState S, const int* cells, const unsigned char* rd_cur, int m) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j >= m) return;
  const int r = cells[j];
  const unsigned char cur = rd_cur[j];
  const int nf = G.ncface[r];
  double cid = 0.0, vs = 0.0;
  for (int k = 0; k < nf; ++k) {
    const int c = G.nb[fidx(G, k, r)];
    const double w = G.iwet[c];
    const double vc = ((cur >> k) & 1) ? S.vis[c] : S.vis1[c];
    cid = cid + w;
    vs = vs + (vc - G.cviscon) * w;
  }
  S.vis[r] = G.cviscon + vs / (cid + 1.0e-15);
}

// a[idx[j]] = vals[j]
// Water levels of a tidal/harmonic string (bnd_eval, boundaries.F90:4098-4124)
// at thrs hours: wse_j = sum_k f_k amp_k cos(speed_k thrs + vu_k - phase_k +
// psi_jk) + offset + wsevar_j, coef [ntc][5] = (f, amp, speed, vu, phase).
__global__ void kf_tide_eval(int nth, int ntc, const double* __restrict__ coef, const double* __restrict__ psi,
                             const double* __restrict__ wsevar, double thrs, double offset, double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nth) return;
  double w = 0.0;
  for (int k = 0; k < ntc; ++k) {
    const double* c = coef + 5 * k;
    w = w + c[0] * c[1] * cos(c[2] * thrs + c[3] - c[4] + psi[(size_t)j * ntc + k]);
  }
  out[j] = w + offset + wsevar[j];
}

__global__ void kf_scatter_vals(const int* idx, const double* vals, int m, double* a) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j < m) a[idx[j]] = vals[j];
}

// string dummies take the value of their cell (bndcopy2ghost, boundaries.F90:4417-4437)
__global__ void kf_copy_to_dummy(const int* cells, const int* dummies, int m, double* a) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j < m) a[dummies[j]] = a[cells[j]];
}

// velface_eta (flow_imp.F90:1245-1573), Cartesian/telescoping branch
__global__ void __launch_bounds__(TPB) kf_velface_eta(FlowDev G, FlowState S) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  if (S.h[r] > G.hmin && G.iwet[r] == 1) {
    double umin = 1e6, umax = -1e6, vmin = 1e6, vmax = -1e6;
    const int nf = G.ncface[r];
    for (int k = 0; k < nf; ++k) {
      const int f = fidx(G, k, r);
      const double vel = S.flux[f] / (S.hk[f] * G.ds[f]);
      const int d = G.dir[f];
      const double uf = fnxd(d) * vel, vf = fnyd(d) * vel;
      umin = fmin(umin, uf); umax = fmax(umax, uf);
      vmin = fmin(vmin, vf); vmax = fmax(vmax, vf);
    }
    const double u = fmin(fmax(S.u[r], umin), umax), v = fmin(fmax(S.v[r], vmin), vmax);
    S.u[r] = u; S.v[r] = v;
    S.eta[r] = S.p[r] * G.gravinv;
    S.uv[r] = sqrt(u * u + v * v);
  } else {
    S.h[r] = fmax(G.hmin, S.h[r]);
    S.u[r] = 0.0; S.v[r] = 0.0; S.uv[r] = 0.0; S.eta[r] = -999.0;
  }
}

// flow_convflux (flow.F90:1879-1909), for a hot start: face fluxes from the
// cell velocities on each cell's no-repeat faces, copied with the opposite
// sign to the neighbour's face.  Correctly rounded steps in the reference's
// order: from the same inputs the result equals the host computation's.
__global__ void __launch_bounds__(TPB) kf_convflux(FlowDev G, FlowState S) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  const unsigned char own = G.owned[r];
  for (int k = 0; k < G.ncface[r]; ++k) {
    if (!((own >> k) & 1)) continue;
    const int f = fidx(G, k, r), nck = G.nb[f], d = G.dir[f];
    const double fx = fnxd(d), fy = fnyd(d);
    const double uni = __dadd_rn(__dmul_rn(fx, S.u[r]), __dmul_rn(fy, S.v[r]));
    const double unk = __dadd_rn(__dmul_rn(fx, S.u[nck]), __dmul_rn(fy, S.v[nck]));
    const double fk = G.fintp[f];
    const double w = (double)(G.iwet[r] * G.iwet[nck]);
    const double fl = __dmul_rn(__dmul_rn(__dmul_rn(w, G.ds[f]), S.hk[f]),
                                __dadd_rn(__dmul_rn(fk, unk), __dmul_rn(__dsub_rn(1.0, fk), uni)));
    S.flux[f] = fl;
    S.flux[fidx(G, G.back[f], nck)] = -fl;
  }
}

// flow_update (CMS_Flow.f90:243-300): time levels; pp and its gradient reset
__global__ void __launch_bounds__(TPB) kf_update(FlowDev G, FlowState S, double* dppx0, double* dppy0, double* dppx1,
                                                 double* dppy1) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.nD) return;
  S.u1[r] = S.u[r]; S.v1[r] = S.v[r]; S.p1[r] = S.p[r]; S.h1[r] = S.h[r];
  S.pp[r] = 0.0;
  dppx0[r] = 0.0; dppy0[r] = 0.0; dppx1[r] = 0.0; dppy1[r] = 0.0;
}

// Solve prologue on device-order face arrays (solvers.f90:230-240): the same
// arithmetic as k_prologue with acoef read slot-major from the flow state.
template <typename TS>
__global__ void __launch_bounds__(TPB) kf_solve_prologue(FlowDev G, const double* __restrict__ acoef, double* ss,
                                                         const double* __restrict__ sp, double* __restrict__ res,
                                                         const double* __restrict__ phi,
                                                         const signed char* __restrict__ fslot_dev, double relax,
                                                         double* __restrict__ aoff, double* __restrict__ diag,
                                                         double* __restrict__ b, double* __restrict__ x,
                                                         TS* __restrict__ aoff2, TS* __restrict__ diag2,
                                                         double* partials, DevState* st) {
  double v[1] = {0.0};
  for (int r = blockIdx.x * TPB + threadIdx.x; r < G.n; r += gridDim.x * TPB) {
    const double rinv = 1.0 / relax, relaxm = 1.0 - relax;
    const int nf = G.ncface[r];
    const double phir = phi[r];
    double sa = 0.0, sn = 0.0, gh = 0.0;
    for (int k = 0; k < nf; ++k) {
      const int f = fidx(G, k, r);
      const double a = acoef[f];
      const int c = G.nb[f];
      const double pn = phi[c];
      sa = sa + a;
      sn = sn + a * pn;
      const int s = fslot_dev[k * G.n + r];
      if (s >= 0) {
        aoff[(size_t)s * G.n + r] = a;
        if (aoff2) aoff2[(size_t)s * G.n + r] = (TS)a;
      } else {
        gh = gh + a * pn;
      }
    }
    const double ap = (sa - sp[r]) * rinv;
    const double ssr = ss[r] + relaxm * phir * ap;
    ss[r] = ssr;
    const double rr = G.iwet[r] * (sn + ssr - ap * phir) / ap;
    res[r] = rr;
    diag[r] = ap;
    if (diag2) diag2[r] = (TS)ap;
    b[r] = ssr + gh;
    x[r] = phir;
    v[0] += rr * rr;
  }
  if (grid_sum<1>(v, partials, &st->ticket[0])) st->s[S_RMOM] = sqrt(v[0] / (double)G.n);
}

__global__ void __launch_bounds__(TPB) kf_copy(int n, const double* __restrict__ a, double* __restrict__ b) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r < n) b[r] = a[r];
}

// non-finite scan of the water level (sets flag[1])
__global__ void __launch_bounds__(TPB) kf_check(FlowDev G, FlowState S) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r < G.n && !(isfinite(S.p[r]) && isfinite(S.u[r]) && isfinite(S.v[r]))) S.flag[1] = 1;
}

// ---- wetting and drying --------------------------------------------------

// Depth classes of every cell from the water level (the inputs of the wet/dry
// rules, flow.F90:1259-1271 and 1363-1416); a cell whose classes differ from
// the stored ones stores the new ones, raises flag[2] and appends itself to
// S.chg (count in flag[3]; at most one entry per cell per launch).
__global__ void __launch_bounds__(TPB) kf_wet_codes(FlowDev G, FlowState S, unsigned char* code) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.nD) return;
  const double h = depth_of(G, S.p[r], G.zb[r]);
  const unsigned char c = (unsigned char)((h >= G.hdry ? 1 : 0) | (h < G.hdry1 ? 2 : 0) | (h < G.hdry2 ? 4 : 0));
  if (c != code[r]) {
    code[r] = c;
    S.flag[2] = 1;
    S.chg[atomicAdd(&S.flag[3], 1)] = r | ((int)c << 28);
  }
}

// Zero flux and viscosity on the faces of the listed cells that have a dry
// side (flow.F90:1501-1524), both sides of each face.  Listing the cells that
// became dry (and the cells of dummies that did) reaches every face the
// reference zeroes that is not zero already: the flow step leaves flux and
// viscosity zero on faces with a dry side.
__global__ void __launch_bounds__(TPB) kf_wet_faces_list(FlowDev G, FlowState S, const int* list, int m) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j >= m) return;
  const int r = list[j];
  const int nf = G.ncface[r];
  for (int k = 0; k < nf; ++k) {
    const int f = fidx(G, k, r), nck = G.nb[f];
    if (G.iwet[r] * G.iwet[nck] != 0) continue;
    const int fb = fidx(G, G.back[f], nck);
    S.flux[f] = 0.0; S.visk[f] = 0.0;
    S.flux[fb] = 0.0; S.visk[fb] = 0.0;
  }
}

// Zero flux and viscosity on every face with a dry side (flow.F90:1501-1524),
// owned faces mirrored.
__global__ void __launch_bounds__(TPB) kf_wet_faces(FlowDev G, FlowState S) {
  const int r = blockIdx.x * TPB + threadIdx.x;
  if (r >= G.n) return;
  const unsigned char own = G.owned[r];
  const int nf = G.ncface[r];
  const int wr = G.iwet[r];
  for (int k = 0; k < nf; ++k) {
    if (!((own >> k) & 1)) continue;
    const int f = fidx(G, k, r), nck = G.nb[f];
    if (wr * G.iwet[nck] != 0) continue;
    const int fb = fidx(G, G.back[f], nck);
    S.flux[f] = 0.0; S.visk[f] = 0.0;
    S.flux[fb] = 0.0; S.visk[fb] = 0.0;
  }
}

// keeps stencil entries with |w| > 1e-8 in order (screen_weights,
// der_lib.f90:681-715) into slots [q * n + r]; returns the count
__device__ __forceinline__ int gw_keep(int nt, const double* w, const int* idx, int n, int r, int* oi, double* ow) {
  int c = 0;
  for (int k = 0; k <= nt; ++k)
    if (fabs(w[k]) > 1.0e-8) {
      oi[c * n + r] = idx[k];
      ow[c * n + r] = w[k];
      ++c;
    }
  return c;
}

// Wet-cell gradient operator of the listed active cells (all when list is
// null) from the current wet set: der_grad_cbgg (der_lib.f90:272-378) and, for
// joint cells, der_grad_cbggcr (381-443).  Every product and sum is rounded
// on its own, as in the host and reference arithmetic, so the weights are the
// same bits the host would form.
__global__ void __launch_bounds__(TPB) kf_gw_rows(FlowDev G, GWOut O, const int* list, int m) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j >= m) return;
  const int r = list ? list[j] : j;
  const int n = G.n, nmf = G.nmf;
  if (G.iwet[r] == 0) {
    O.ncx[r] = 0; O.ncy[r] = 0;
    O.ngx[r] = 0; O.ngy[r] = 0;
    return;
  }
  double tx[9], ty[9];
  int ti[9], tj[9];
  const int nf = G.ncface[r];
  for (int k = 0; k <= nmf; ++k) { tx[k] = 0.0; ty[k] = 0.0; ti[k] = r; tj[k] = r; }
  const double area = G.areap[r];
  for (int k = 0; k < nf; ++k) {
    const int f = fidx(G, k, r), c = G.nb[f], d = G.dir[f];
    const double dsx = fnxd(d) * G.ds[f], dsy = fnyd(d) * G.ds[f], fk = G.fintp[f];
    ti[k + 1] = c; tj[k + 1] = c;
    if (G.iwet[c] == 1) {
      const double fp = __dsub_rn(1.0, fk);
      tx[0] = __dadd_rn(tx[0], __dmul_rn(dsx, fp));
      tx[k + 1] = __dmul_rn(dsx, fk);
      ty[0] = __dadd_rn(ty[0], __dmul_rn(dsy, fp));
      ty[k + 1] = __dmul_rn(dsy, fk);
    } else {
      tx[0] = __dadd_rn(tx[0], dsx);
      ty[0] = __dadd_rn(ty[0], dsy);
    }
  }
  for (int k = 0; k <= nmf; ++k) { tx[k] = __ddiv_rn(tx[k], area); ty[k] = __ddiv_rn(ty[k], area); }
  const int cx = gw_keep(nmf, tx, ti, n, r, O.icx, O.wcx);
  const int cy = gw_keep(nmf, ty, tj, n, r, O.icy, O.wcy);
  double sx = 0.0, sy = 0.0;
  for (int q = 0; q < cx; ++q) sx = __dadd_rn(sx, O.wcx[q * n + r]);
  for (int q = 0; q < cy; ++q) sy = __dadd_rn(sy, O.wcy[q * n + r]);
  const double mx = __ddiv_rn(sx, (double)cx), my = __ddiv_rn(sy, (double)cy);
  for (int q = 0; q < cx; ++q) O.wcx[q * n + r] = __dsub_rn(O.wcx[q * n + r], mx);
  for (int q = 0; q < cy; ++q) O.wcy[q * n + r] = __dsub_rn(O.wcy[q * n + r], my);
  O.ncx[r] = cx; O.ncy[r] = cy;
  if (G.ider != 2 || !G.joint[r]) return;
  const unsigned char own = G.owned[r], cr = G.crmask[r];
  for (int k = 0; k <= nmf; ++k) { tx[k] = 0.0; ty[k] = 0.0; ti[k] = 0; tj[k] = 0; }
  ti[0] = r; tj[0] = r;
  for (int k = 0; k < nf; ++k) {
    if (!((own >> k) & 1)) continue;
    const int f = fidx(G, k, r), c = G.nb[f], d = G.dir[f];
    const bool xface = (d == 2 || d == 4);
    if (!xface) tj[k + 1] = c;
    if (!((cr >> k) & 1) || G.iwet[c] == 0) continue;
    const int fb = fidx(G, G.back[f], c);
    const double fk = G.fintp[f], fp = __dsub_rn(1.0, fk);
    if (xface) {
      const double dsx = fnxd(d) * G.ds[f];
      tx[0] = __dadd_rn(tx[0], __ddiv_rn(__dmul_rn(__dmul_rn(dsx, fp), G.rpy[f]), area));
      tx[k + 1] = __ddiv_rn(__dmul_rn(__dmul_rn(dsx, fk), G.rpy[fb]), area);
      ti[k + 1] = c;
    } else {
      const double dsy = fnyd(d) * G.ds[f];
      ty[0] = __dadd_rn(ty[0], __ddiv_rn(__dmul_rn(__dmul_rn(dsy, fp), G.rpx[f]), area));
      ty[k + 1] = __ddiv_rn(__dmul_rn(__dmul_rn(dsy, fk), G.rpx[fb]), area);
    }
  }
  O.ngx[r] = gw_keep(nmf, tx, ti, n, r, O.igx, O.wgxy);
  O.ngy[r] = gw_keep(nmf, ty, tj, n, r, O.igy, O.wgyx);
}

// buf[3j..3j+2] = (u, v, vis) of cell idx[j]
__global__ void kf_gather_uvv(const int* idx, int m, const double* u, const double* v, const double* vis,
                              double* buf) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j >= m) return;
  const int c = idx[j];
  buf[3 * j] = u[c]; buf[3 * j + 1] = v[c]; buf[3 * j + 2] = vis[c];
}

// (u, v, vis) of cell idx[j] = buf[3j..3j+2]
__global__ void kf_scatter_uvv(const int* idx, int m, const double* buf, double* u, double* v, double* vis) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j >= m) return;
  const int c = idx[j];
  u[c] = buf[3 * j]; v[c] = buf[3 * j + 1]; vis[c] = buf[3 * j + 2];
}

// a[idx[j]] = v[j] (bytes)
__global__ void kf_scatter_u8(const int* idx, const unsigned char* v, int m, unsigned char* a) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j < m) a[idx[j]] = v[j];
}

// a[idx[j]] = v[j] (ints)
__global__ void kf_scatter_i32(const int* idx, const int* v, int m, int* a) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j < m) a[idx[j]] = v[j];
}

// ---- flow_pond on the device (flow.F90:1807-1876): connected components of
// the wet active cells by union-find.  A root is only ever hooked under a
// root of smaller index (compare-and-swap), and path halving only points a
// cell at an ancestor, so a parent always has a smaller index than its child:
// every walk up a chain ends, and the partition does not depend on the order
// in which threads meet.  The walks are bounded all the same.

constexpr int kUfLimit = 1 << 26;

__device__ __forceinline__ int uf_root(int* par, int x) {
  for (int guard = 0; guard < kUfLimit; ++guard) {
    const int p = par[x];
    if (p == x) return x;
    const int gp = par[p];
    if (gp != p) par[x] = gp;
    x = p;
  }
  return x;
}

__device__ __forceinline__ void uf_union(int* par, int a, int b) {
  int ra = uf_root(par, a), rb = uf_root(par, b);
  for (int guard = 0; guard < kUfLimit && ra != rb; ++guard) {
    if (ra < rb) { const int t = ra; ra = rb; rb = t; }
    const int old = atomicCAS(&par[ra], ra, rb);
    if (old == ra) return;
    ra = uf_root(par, old);
    rb = uf_root(par, rb);
  }
}

__global__ void __launch_bounds__(TPB) kf_pond_init(int n, int* par) {
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i < n) par[i] = i;
}

// union of every pair of face neighbours that are both wet active cells of pn
__global__ void __launch_bounds__(TPB) kf_pond_hook(FlowDev G, const unsigned char* pn, int* par) {
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= G.n || !pn[i]) return;
  const int nf = G.ncface[i];
  for (int k = 0; k < nf; ++k) {
    const int j = G.nb[fidx(G, k, i)];
    if (j > i && j < G.n && pn[j]) uf_union(par, i, j);
  }
}

// components holding a wet string cell are kept
__global__ void kf_pond_seed(const int* seeds, int m, const unsigned char* pn, int* par, unsigned char* seeded) {
  const int j = blockIdx.x * TPB + threadIdx.x;
  if (j >= m) return;
  const int s = seeds[j];
  if (pn[s]) seeded[uf_root(par, s)] = 1;
}

// final wet flags of the active cells (pn, less the unseeded components when
// ponding is off); cells whose flag changed are appended to chg (count in cnt)
__global__ void __launch_bounds__(TPB) kf_pond_final(int n, const unsigned char* pn, int* par,
                                                     const unsigned char* seeded, int ponding, int* iwet, int* chg,
                                                     int* cnt) {
  const int i = blockIdx.x * TPB + threadIdx.x;
  if (i >= n) return;
  const int w = pn[i] && (ponding || seeded[uf_root(par, i)]) ? 1 : 0;
  if (w != iwet[i]) {
    iwet[i] = w;
    chg[atomicAdd(cnt, 1)] = i;
  }
}

}  // namespace cms
