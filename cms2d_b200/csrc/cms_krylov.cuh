// Device kernels of the preconditioned Krylov solves (device order, ELL layout).
//
// Matrix: A = diag(ap) - O, O >= 0 the face coefficients acoef(k,i) between
// active cells (source/solvers/pbicgstab.f90:59, pgmres.f90:164-165).
// Storage, device row r of n:
//   aoff[s*n + r]  coefficient of ELL slot s (lower slots 0..KL-1, upper
//                  KL..KL+KU-1, padding = 0 with col = r);
//   col [s*n + r]  device column of the slot;
//   diag[r]        ap;
//   luoff / invd   the ILU(0) factor: signed multipliers l_rj in lower slots,
//                  signed u_rk in upper slots, invd = 1/u_rr (the MSR layout
//                  of ilu0.f90 with alu(i) = 1/u_ii).
#pragma once
#include "cms_common.cuh"

namespace cms {

// ----------------------------------------------------------------------------
// solve() prologue, natural order (source/solvers/solvers.f90:230-240):
//   ap = (sum_k acoef - sp)/relax;  ss += (1-relax)*phi*ap;
//   res = iwet*(sum_k acoef*phi_nb + ss - ap*phi)/ap;  rmom = sqrt(sum res^2/n)
// and the scatter of the system into device order: diag, ELL slots, right-hand
// side b = ss + sum over dummy neighbours of acoef*phi_dummy, x = phi.  A
// second copy of the matrix in type TS is written when aoff2 != nullptr.
template <typename T, typename TS>
__global__ void __launch_bounds__(TPB) k_prologue(int n, int nmf, const T* __restrict__ acoef, T* __restrict__ ss,
                                                  const T* __restrict__ sp, T* __restrict__ res,
                                                  const T* __restrict__ phi, const int* __restrict__ c2c,
                                                  const int* __restrict__ ncface, const int* __restrict__ iwet,
                                                  const signed char* __restrict__ fslot,
                                                  const int* __restrict__ iperm, T relax, T* __restrict__ aoff,
                                                  T* __restrict__ diag, T* __restrict__ b, T* __restrict__ x,
                                                  TS* __restrict__ aoff2, TS* __restrict__ diag2,
                                                  double* partials, DevState* st) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    const T rinv = T(1) / relax;
    const T relaxm = T(1) - relax;
    const int nf = ncface[i];
    const T phii = phi[i];
    const int r = iperm[i];
    T sa = T(0), sn = T(0), gh = T(0);
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
      if (k < nf) {
        const T a = acoef[(size_t)i * nmf + k];
        const int c = c2c[(size_t)i * nmf + k] - 1;
        const T pn = phi[c];
        sa = sa + a;
        sn = sn + a * pn;
        const int s = fslot[(size_t)i * nmf + k];
        if (s >= 0) {
          aoff[(size_t)s * n + r] = a;
          if (aoff2) aoff2[(size_t)s * n + r] = (TS)a;
        } else {
          gh = gh + a * pn;
        }
      }
    }
    const T ap = (sa - sp[i]) * rinv;
    const T ssi = ss[i] + relaxm * phii * ap;
    ss[i] = ssi;
    const T resi = T(iwet[i]) * (sn + ssi - ap * phii) / ap;
    res[i] = resi;
    diag[r] = ap;
    if (diag2) diag2[r] = (TS)ap;
    b[r] = ssi + gh;
    x[r] = phii;
    v[0] += (double)resi * (double)resi;
  }
  if (grid_sum<1>(v, partials, &st->ticket[0])) {
    st->s[S_RMOM] = sqrt(v[0] / (double)n);
  }
}

// x (device order) -> phi (natural order)
template <typename TD, typename TS>
__global__ void __launch_bounds__(TPB) k_scatter(int n, const int* __restrict__ perm, const TS* __restrict__ x,
                                                 TD* __restrict__ phi) {
  for (int r = blockIdx.x * TPB + threadIdx.x; r < n; r += gridDim.x * TPB) phi[perm[r]] = (TD)x[r];
}

// ----------------------------------------------------------------------------
// ILU(0) of the rows of one group (ilu0.f90:22-62 restated per row): rows of
// earlier groups are final.  For each lower entry j in ascending column order:
// l = a_rj / u_jj; then every upper entry (j,k) of row j updates the diagonal
// (k == r) or an entry of row r with the same column.
template <typename T>
__global__ void __launch_bounds__(TPB) k_ilu0(int n, int r0, int r1, int KL, int klg, int kug,
                                              const int* __restrict__ col, const signed char* __restrict__ nlo,
                                              const signed char* __restrict__ nup, const T* __restrict__ aoff,
                                              const T* __restrict__ diag, T* luoff, T* invd) {
 for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
  const int kl = min(klg, (int)nlo[r]), ku = min(kug, (int)nup[r]);
  T al[KMAX], au[KMAX];
  int cl[KMAX], cu[KMAX];
#pragma unroll
  for (int s = 0; s < KMAX; ++s) {
    if (s < kl) { cl[s] = col[(size_t)s * n + r]; al[s] = -aoff[(size_t)s * n + r]; }
    else { cl[s] = r; al[s] = T(0); }
    if (s < ku) { cu[s] = col[(size_t)(KL + s) * n + r]; au[s] = -aoff[(size_t)(KL + s) * n + r]; }
    else { cu[s] = r; au[s] = T(0); }
  }
  T d = diag[r];
#pragma unroll
  for (int s = 0; s < KMAX; ++s) {
    if (s < kl) {
      const int j = cl[s];
      if (j == r) { al[s] = T(0); continue; }
      const T lij = al[s] * invd[j];
      al[s] = lij;
      const int nuj = nup[j];
#pragma unroll 1
      for (int t2 = 0; t2 < nuj; ++t2) {
        const int k = col[(size_t)(KL + t2) * n + j];
        if (k == j) continue;
        const T ujk = luoff[(size_t)(KL + t2) * n + j];
        if (k == r) {
          d = d - lij * ujk;
        } else {
#pragma unroll
          for (int s2 = s + 1; s2 < KMAX; ++s2)
            if (s2 < kl && cl[s2] == k) al[s2] = al[s2] - lij * ujk;
#pragma unroll
          for (int t = 0; t < KMAX; ++t)
            if (t < ku && cu[t] == k) au[t] = au[t] - lij * ujk;
        }
      }
    }
  }
  invd[r] = T(1) / d;
#pragma unroll
  for (int s = 0; s < KMAX; ++s) {
    if (s < kl) luoff[(size_t)s * n + r] = al[s];
    if (s < ku) luoff[(size_t)(KL + s) * n + r] = au[s];
  }
 }
}

// ----------------------------------------------------------------------------
// Forward sweep of one group: z_r = y_r - sum_{lower} l_rj z_j (lusol,
// sparse.f90:248-253).  The right-hand side y is formed in place:
enum FwdMode : int {
  FWD_PLAIN = 0,    // y = yin
  FWD_BICG_P = 1,   // p = r + omg*(p - alf*u); y = p            (pbicgstab.f90:44-51)
  FWD_BICG_R = 2,   // x += gam*z_old; r -= gam*u; y = r          (pbicgstab.f90:67-70)
  FWD_GM_SCALE = 3, // v_i *= scale_i (stored back); y = v_i      (pgmres.f90:150,178)
  FWD_GM_COMB = 4   // y = sum_{j<=i} v_j * y_j                   (pgmres.f90:219-221)
};

struct GmVecs {
  void* v[5];  // v_1..v_4 at index 1..4
};

template <typename T, int MODE>
__global__ void __launch_bounds__(TPB) k_fwd(int n, int r0, int r1, int klg, int step, const int* __restrict__ col,
                                             const signed char* __restrict__ nlo, const T* __restrict__ luoff, T* z,
                                             const T* __restrict__ yin, T* p, T* r_, const T* __restrict__ u, T* x,
                                             GmVecs gv, const DevState* st) {
  if (st->done) return;
  if (MODE == FWD_GM_SCALE && !st->active) return;
 for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
  const int kl = klg > 0 ? (int)nlo[r] : 0;
  T y;
  if (MODE == FWD_PLAIN) {
    y = yin[r];
  } else if (MODE == FWD_BICG_P) {
    // scalars are formed in FP64 (an FP32 solve of a tiny right-hand side
    // would otherwise underflow them to 0/0) and applied in T
    const double bet = st->s[S_BET], gam = st->s[S_GAM], alfd = st->s[S_ALF], bet0 = st->s[S_BET0];
    const T omg = (T)(bet * gam / (alfd * bet0 + SMALL));
    const T alf = (T)alfd;
    y = r_[r] + omg * (p[r] - alf * u[r]);
    p[r] = y;
  } else if (MODE == FWD_BICG_R) {
    const T gam = (T)st->s[S_GAM];
    x[r] = x[r] + gam * z[r];
    y = r_[r] - gam * u[r];
    r_[r] = y;
  } else if (MODE == FWD_GM_SCALE) {
    T* vi = (T*)gv.v[step];
    y = (T)st->s[S_SCALE1 + step - 1] * vi[r];
    vi[r] = y;
  } else {  // FWD_GM_COMB
    const int ni = st->ifinal;
    y = T(0);
#pragma unroll
    for (int j = 1; j <= 3; ++j)
      if (j <= ni) y = y + ((const T*)gv.v[j])[r] * (T)st->s[S_Y + j];
  }
  T acc = y;
#pragma unroll
  for (int s = 0; s < KMAX; ++s)
    if (s < kl) acc = acc - luoff[(size_t)s * n + r] * z[col[(size_t)s * n + r]];
  z[r] = acc;
 }
}

// Backward sweep of one group: z_r = invd_r * (z_r - sum_{upper} u_rk z_k)
// (sparse.f90:256-261); FINAL also adds the result to x (pgmres.f90:226).
template <typename T, bool FINAL>
__global__ void __launch_bounds__(TPB) k_bwd(int n, int r0, int r1, int KL, int kug, const int* __restrict__ col,
                                             const signed char* __restrict__ nup, const T* __restrict__ luoff,
                                             const T* __restrict__ invd, T* z, T* x, int need_active,
                                             const DevState* st) {
  if (st->done) return;
  if (need_active && !st->active) return;
 for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
  const int ku = kug > 0 ? (int)nup[r] : 0;
  T acc = z[r];
#pragma unroll
  for (int t = 0; t < KMAX; ++t)
    if (t < ku) acc = acc - luoff[(size_t)(KL + t) * n + r] * z[col[(size_t)(KL + t) * n + r]];
  const T zr = invd[r] * acc;
  z[r] = zr;
  if (FINAL) x[r] = x[r] + zr;
 }
}

// ----------------------------------------------------------------------------
// y = A z over all rows (group table), fused with the dot products the Krylov
// recurrences need next.  The last block updates the scalars.
enum SpmvMode : int {
  SPMV_BICG_U = 0,  // u = A z; ukr0 = u.r0; gam = bet/ukr0; bet0 = bet   (pbicgstab.f90:56-63)
  SPMV_BICG_V = 1,  // v = A z; sum1 = v.r; sum2 = v.v; alf = sum1/max(sum2,small)  (76-84)
  SPMV_GM = 2       // w = A z; hh(1,i) = v_1.w                          (pgmres.f90:163-172)
};

template <typename T, int MODE>
__global__ void __launch_bounds__(TPB) k_spmv(int n, int KL, GroupTab tab, int step, const int* __restrict__ col,
                                              const signed char* __restrict__ nlo,
                                              const signed char* __restrict__ nup, const T* __restrict__ aoff,
                                              const T* __restrict__ diag, const T* __restrict__ z,
                                              T* __restrict__ y, const T* __restrict__ d1, double* partials,
                                              DevState* st) {
  if (st->done) return;
  if (MODE == SPMV_GM && !st->active) return;
  const int g = tab_group(tab, blockIdx.x);
  const int stride = (tab.blk[g + 1] - tab.blk[g]) * TPB;
  double v[MODE == SPMV_BICG_V ? 2 : 1];
#pragma unroll
  for (int q = 0; q < (MODE == SPMV_BICG_V ? 2 : 1); ++q) v[q] = 0.0;
  for (int r = tab.start[g] + (blockIdx.x - tab.blk[g]) * TPB + threadIdx.x; r < tab.start[g + 1]; r += stride) {
    const int kl = tab.kl[g] > 0 ? (int)nlo[r] : 0, ku = tab.ku[g] > 0 ? (int)nup[r] : 0;
    T sum = T(0);
#pragma unroll
    for (int s = 0; s < KMAX; ++s)
      if (s < kl) sum = sum + aoff[(size_t)s * n + r] * z[col[(size_t)s * n + r]];
#pragma unroll
    for (int t = 0; t < KMAX; ++t)
      if (t < ku) sum = sum + aoff[(size_t)(KL + t) * n + r] * z[col[(size_t)(KL + t) * n + r]];
    const T yr = diag[r] * z[r] - sum;
    y[r] = yr;
    if (MODE == SPMV_BICG_U) v[0] += (double)yr * (double)d1[r];
    if (MODE == SPMV_BICG_V) { v[0] += (double)yr * (double)d1[r]; v[1] += (double)yr * (double)yr; }
    if (MODE == SPMV_GM) v[0] += (double)d1[r] * (double)yr;
  }
  if (grid_sum(v, partials, &st->ticket[1])) {
    if (MODE == SPMV_BICG_U) {
      st->s[S_UKR0] = v[0];
      st->s[S_GAM] = st->s[S_BET] / v[0];
      st->s[S_BET0] = st->s[S_BET];
    } else if (MODE == SPMV_BICG_V) {
      st->s[S_SUM1] = v[0];
      st->s[S_SUM2] = v[1];
      st->s[S_ALF] = v[0] / fmax(v[1], SMALL);
    } else {
      st->s[S_HH + 0 * 3 + (step - 1)] = v[0];
    }
  }
}

// ----------------------------------------------------------------------------
// BiCGStab start (pbicgstab.f90:20-38): r = b - A x + small, r0 = r, p=u=v=0,
// res0 = sum|r0| (norm 1) or ||r0||_2 (norm 2), bet = r.r0.  xzero: x = 0.
template <typename T>
__global__ void __launch_bounds__(TPB) k_bicg_init(int n, int KL, GroupTab tab, int xzero, int maxit, int norm,
                                                   double tol, const int* __restrict__ col,
                                                   const signed char* __restrict__ nlo,
                                                   const signed char* __restrict__ nup, const T* __restrict__ aoff,
                                                   const T* __restrict__ diag, const T* __restrict__ b, T* x, T* r_,
                                                   T* r0, T* p, T* u, T* v_, double* partials, DevState* st) {
  const int g = tab_group(tab, blockIdx.x);
  const int stride = (tab.blk[g + 1] - tab.blk[g]) * TPB;
  double v[2] = {0.0, 0.0};
  for (int r = tab.start[g] + (blockIdx.x - tab.blk[g]) * TPB + threadIdx.x; r < tab.start[g + 1]; r += stride) {
    T term;
    if (xzero) {
      x[r] = T(0);
      term = b[r];
    } else {
      const int kl = tab.kl[g] > 0 ? (int)nlo[r] : 0, ku = tab.ku[g] > 0 ? (int)nup[r] : 0;
      T sum = T(0);
#pragma unroll
      for (int s = 0; s < KMAX; ++s)
        if (s < kl) sum = sum + aoff[(size_t)s * n + r] * x[col[(size_t)s * n + r]];
#pragma unroll
      for (int t = 0; t < KMAX; ++t)
        if (t < ku) sum = sum + aoff[(size_t)(KL + t) * n + r] * x[col[(size_t)(KL + t) * n + r]];
      term = sum + b[r] - diag[r] * x[r];
    }
    const T rr = term + (T)SMALL;
    r_[r] = rr;
    r0[r] = rr;
    p[r] = T(0);
    u[r] = T(0);
    v_[r] = T(0);
    v[0] += fabs((double)rr);
    v[1] += (double)rr * (double)rr;
  }
  if (grid_sum(v, partials, &st->ticket[2])) {
    st->s[S_RES0] = (norm == 1) ? v[0] : sqrt(v[1]);
    st->s[S_BET] = v[1];
    st->s[S_ALF] = 1.0;
    st->s[S_BET0] = 1.0;
    st->s[S_GAM] = 1.0;
    st->s[S_TOL] = tol;
    st->s[S_RELRES] = 1.0;
    st->iter = 0;
    st->maxit = maxit;
    st->norm = norm;
    st->converged = 0;
    st->nonfinite = 0;
    st->active = 0;
    st->done = (maxit <= 0) ? 1 : 0;
  }
}

// x += alf z; r -= alf v; stopping test on sum|r| (or ||r||_2) / res0; next
// bet = r.r0 (pbicgstab.f90:87-95 and 42-43).
template <typename T>
__global__ void __launch_bounds__(TPB) k_bicg_update(int n, const T* __restrict__ z, const T* __restrict__ v_,
                                                     T* __restrict__ x, T* __restrict__ r_,
                                                     const T* __restrict__ r0, double* partials, DevState* st) {
  if (st->done) return;
  double v[3] = {0.0, 0.0, 0.0};
  const T alf = (T)st->s[S_ALF];
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    x[i] = x[i] + alf * z[i];
    const T ri = r_[i] - alf * v_[i];
    r_[i] = ri;
    v[0] += fabs((double)ri);
    v[1] += (double)ri * (double)ri;
    v[2] += (double)ri * (double)r0[i];
  }
  if (grid_sum(v, partials, &st->ticket[3])) {
    st->iter += 1;
    const double res = (st->norm == 1) ? v[0] : sqrt(v[1]);
    const double rel = res / st->s[S_RES0];
    st->s[S_RES] = res;
    st->s[S_RELRES] = rel;
    st->s[S_BET] = v[2];
    if (!isfinite(rel)) { st->nonfinite = 1; st->done = 1; }
    else if (rel < st->s[S_TOL]) { st->converged = 1; st->done = 1; }
    else if (st->iter >= st->maxit) { st->done = 1; }
  }
}

// ----------------------------------------------------------------------------
// GMRES(3) (pgmres.f90): restart residual v_1 = b - A x, ro = sqrt(sum v_1^2 + small)
template <typename T>
__global__ void __launch_bounds__(TPB) k_gm_resid(int n, int KL, GroupTab tab, const int* __restrict__ col,
                                                  const signed char* __restrict__ nlo,
                                                  const signed char* __restrict__ nup, const T* __restrict__ aoff,
                                                  const T* __restrict__ diag, const T* __restrict__ b,
                                                  const T* __restrict__ x, T* __restrict__ v1, double* partials,
                                                  DevState* st) {
  if (st->done) return;
  const int g = tab_group(tab, blockIdx.x);
  const int stride = (tab.blk[g + 1] - tab.blk[g]) * TPB;
  double v[1] = {0.0};
  for (int r = tab.start[g] + (blockIdx.x - tab.blk[g]) * TPB + threadIdx.x; r < tab.start[g + 1]; r += stride) {
    const int kl = tab.kl[g] > 0 ? (int)nlo[r] : 0, ku = tab.ku[g] > 0 ? (int)nup[r] : 0;
    T sum = T(0);
#pragma unroll
    for (int s = 0; s < KMAX; ++s)
      if (s < kl) sum = sum + aoff[(size_t)s * n + r] * x[col[(size_t)s * n + r]];
#pragma unroll
    for (int t = 0; t < KMAX; ++t)
      if (t < ku) sum = sum + aoff[(size_t)(KL + t) * n + r] * x[col[(size_t)(KL + t) * n + r]];
    const T vr = sum + b[r] - diag[r] * x[r];
    v1[r] = vr;
    v[0] += (double)vr * (double)vr;
  }
  if (grid_sum(v, partials, &st->ticket[2])) {
    const double ro = sqrt(v[0] + SMALL);
    if (st->iter == 0) {
      st->s[S_EPS11] = st->s[S_TOL] * ro;
      st->s[S_RO0] = ro;
    }
    st->s[S_RO] = ro;
    st->s[S_SCALE1] = 1.0 / (ro + SMALL);
    st->s[S_RS1 + 1] = ro;
    st->active = 1;
    st->ifinal = 0;
    st->stop = 0;
  }
}

// MGS step j of Arnoldi step i: w -= hh(j,i) v_j (skipped when hh == 0, as
// aesmbpak does), then hh(j+1,i) = v_{j+1}.w, or for j == i the norm, the
// Givens update and -- when the cycle ends -- the small triangular solve
// (pgmres.f90:171-215).
template <typename T>
__global__ void __launch_bounds__(TPB) k_mgs(int n, int j, int i, GmVecs gv, double* partials, DevState* st) {
  if (st->done || !st->active) return;
  T* w = (T*)gv.v[i + 1];
  const T* vj = (const T*)gv.v[j];
  const T h = (T)st->s[S_HH + (j - 1) * 3 + (i - 1)];
  double v[1] = {0.0};
  for (int q = blockIdx.x * TPB + threadIdx.x; q < n; q += gridDim.x * TPB) {
    T wq = w[q];
    if (h != T(0)) { wq = wq + (-h) * vj[q]; w[q] = wq; }
    if (j < i) v[0] += (double)((const T*)gv.v[j + 1])[q] * (double)wq;
    else v[0] += (double)wq * (double)wq;
  }
  if (grid_sum(v, partials, &st->ticket[4])) {
    double* s = st->s;
    auto HH = [s](int jj, int ii) -> double& { return s[S_HH + (jj - 1) * 3 + (ii - 1)]; };
    if (j < i) {
      HH(j + 1, i) = v[0];
      return;
    }
    const int i1 = i + 1;
    double t = sqrt(v[0] + SMALL);
    HH(i1, i) = t;
    s[S_SCALE1 + i] = 1.0 / fmax(t, SMALL);
    for (int k = 2; k <= i; ++k) {
      const int k1 = k - 1;
      const double tt = HH(k1, i);
      const double ck = s[S_C + k1], sk = s[S_S + k1];
      HH(k1, i) = ck * tt + sk * HH(k, i);
      HH(k, i) = -sk * tt + ck * HH(k, i);
    }
    double gam = sqrt(HH(i, i) * HH(i, i) + HH(i1, i) * HH(i1, i));
    if (gam == 0.0) gam = SMALL;
    const double ci = HH(i, i) / gam, si = HH(i1, i) / gam;
    s[S_C + i] = ci;
    s[S_S + i] = si;
    s[S_RS1 + i1] = -si * s[S_RS1 + i];
    s[S_RS1 + i] = ci * s[S_RS1 + i];
    HH(i, i) = ci * HH(i, i) + si * HH(i1, i);
    const double ro = fabs(s[S_RS1 + i1]);
    s[S_RO] = ro;
    st->inner += 1;
    if (i < 3 && ro > s[S_EPS11]) return;  // next Arnoldi step
    st->active = 0;
    st->ifinal = i;
    double rs[4];
    for (int k = 1; k <= i; ++k) rs[k] = s[S_RS1 + k];
    rs[i] = rs[i] / HH(i, i);
    for (int ii = 2; ii <= i; ++ii) {
      const int k = i - ii + 1, k1 = k + 1;
      double tt = rs[k];
      for (int jj = k1; jj <= i; ++jj) tt = tt - HH(k, jj) * rs[jj];
      rs[k] = tt / HH(k, k);
    }
    for (int k = 1; k <= i; ++k) s[S_Y + k] = rs[k];
    s[S_RELRES] = (double)ro / s[S_RO0];
    if (!isfinite((double)ro)) { st->nonfinite = 1; st->stop = 1; }
    if (ro <= s[S_EPS11]) st->stop = 1;
  }
}

__global__ void k_gm_cycle_end(DevState* st) {
  if (st->done) return;
  st->iter += 1;
  if (st->stop) {
    st->done = 1;
    st->converged = st->nonfinite ? 0 : 1;
  } else if (st->iter >= st->maxit) {
    st->done = 1;
  }
}

// GMRES state reset at the start of a solve.
__global__ void k_gm_start(DevState* st, int maxit, double tol) {
  st->iter = 0;
  st->inner = 0;
  st->maxit = maxit;
  st->s[S_TOL] = tol;
  st->s[S_RELRES] = 1.0;
  st->converged = 0;
  st->nonfinite = 0;
  st->active = 0;
  st->stop = 0;
  st->ifinal = 0;
  st->done = (maxit <= 0) ? 1 : 0;
}

// ----------------------------------------------------------------------------
// FP64 residual of the device-order system, r = b - A x (all rows), sum r^2
// into S_NRM2 (slot_out).  Optionally stores r (FP64) and its FP32 copy.
template <typename TA, typename TX>
__global__ void __launch_bounds__(TPB) k_resid64(int n, int KL, GroupTab tab, const int* __restrict__ col,
                                                 const signed char* __restrict__ nlo,
                                                 const signed char* __restrict__ nup, const TA* __restrict__ aoff,
                                                 const TA* __restrict__ diag, const double* __restrict__ b,
                                                 const TX* __restrict__ x, double* __restrict__ rout,
                                                 float* __restrict__ rout32, int slot_out, double* partials,
                                                 DevState* st) {
  const int g = tab_group(tab, blockIdx.x);
  const int stride = (tab.blk[g + 1] - tab.blk[g]) * TPB;
  double v[1] = {0.0};
  for (int r = tab.start[g] + (blockIdx.x - tab.blk[g]) * TPB + threadIdx.x; r < tab.start[g + 1]; r += stride) {
    const int kl = tab.kl[g] > 0 ? (int)nlo[r] : 0, ku = tab.ku[g] > 0 ? (int)nup[r] : 0;
    double sum = 0.0;
#pragma unroll
    for (int s = 0; s < KMAX; ++s)
      if (s < kl) sum += (double)aoff[(size_t)s * n + r] * (double)x[col[(size_t)s * n + r]];
#pragma unroll
    for (int t = 0; t < KMAX; ++t)
      if (t < ku) sum += (double)aoff[(size_t)(KL + t) * n + r] * (double)x[col[(size_t)(KL + t) * n + r]];
    const double rr = b[r] - ((double)diag[r] * (double)x[r] - sum);
    if (rout) rout[r] = rr;
    if (rout32) rout32[r] = (float)rr;
    v[0] += rr * rr;
  }
  if (grid_sum(v, partials, &st->ticket[5])) st->s[slot_out] = v[0];
}

// x64 += scale * d32 (refinement correction; scale undoes the normalisation)
__global__ void __launch_bounds__(TPB) k_ir_correct(int n, const float* __restrict__ d, double* __restrict__ x,
                                                    const DevState* st) {
  const double scale = st->s[S_IRSCALE];
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) x[i] += scale * (double)d[i];
}

// Undoes the last correction (the same scale, opposite sign).
__global__ void __launch_bounds__(TPB) k_ir_undo(int n, const float* __restrict__ d, double* __restrict__ x,
                                                 const DevState* st) {
  const double scale = st->s[S_IRSCALE];
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) x[i] -= scale * (double)d[i];
}

// r32 = r64 / ||r64||_2 (the FP32 correction solve sees a unit-norm right-hand side)
__global__ void __launch_bounds__(TPB) k_ir_scale(int n, const double* __restrict__ r, float* __restrict__ r32,
                                                  DevState* st) {
  const double nrm = sqrt(st->s[S_NRM2]);
  const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) r32[i] = (float)(r[i] * inv);
  if (blockIdx.x == 0 && threadIdx.x == 0) st->s[S_IRSCALE] = nrm;
}

template <typename TD, typename TS>
__global__ void __launch_bounds__(TPB) k_convert(int n, const TS* __restrict__ a, TD* __restrict__ b) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) b[i] = (TD)a[i];
}

}  // namespace cms
