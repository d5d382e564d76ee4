// Device kernels of the MATRIX_SOLVER options other than BiCGStab and GMRES
// (source/solvers/solvers.f90:242-289): Gauss-Seidel and its SOR /
// symmetric variants, Stone's SIP, and CG / BiCGStab preconditioned by the
// diagonal incomplete Cholesky factor (ICCG, ICCGSTAB).
//
// All work in device order on the ELL matrix of cms_krylov.cuh (A = diag - O,
// aoff = O >= 0, right-hand side b with the dummy-cell terms folded in).
// Recurrences follow the groups: the rows of a group are not coupled, and
// every coupling of a row to an earlier group is a lower slot.  In the
// natural (level-scheduled) ordering this is the reference's serial loop; in
// the multicolour ordering it is the multicolour form of the same method.
// With few groups (colours) each group is one launch; with many (the natural
// ordering's level sets) the passes run pipelined inside one launch
// (k_gs_pipe, k_tri_pipe below).
//
// Every iteration kernel starts with `if (st->done) return;`, so the host can
// issue a whole solve's launches ahead and let the device stopping test end it.
#pragma once
#include "cms_common.cuh"

namespace cms {

// sum over the row's stored couplings of aoff * x (lower slots, then upper)
template <typename T>
__device__ __forceinline__ T row_off(int n, int KL, int r, int kl, int ku, const int* __restrict__ col,
                                     const T* __restrict__ aoff, const T* x) {
  T t = T(0);
#pragma unroll
  for (int s = 0; s < KMAX; ++s)
    if (s < kl) t = t + aoff[(size_t)s * n + r] * x[col[(size_t)s * n + r]];
#pragma unroll
  for (int s = 0; s < KMAX; ++s)
    if (s < ku) t = t + aoff[(size_t)(KL + s) * n + r] * x[col[(size_t)(KL + s) * n + r]];
  return t;
}

// One Gauss-Seidel pass over a group (gauss-seidel.f90:2-75):
//   x_r = (b_r + sum aoff x) / diag_r,  SOR: w (b_r + sum aoff x) / diag_r + (1-w) x_r.
template <typename T, bool SOR>
__global__ void __launch_bounds__(TPB) k_gs(int n, int r0, int r1, int KL, int klg, int kug,
                                            const int* __restrict__ col, const signed char* __restrict__ nlo,
                                            const signed char* __restrict__ nup, const T* __restrict__ aoff,
                                            const T* __restrict__ diag, const T* __restrict__ b, T* x, T w) {
  for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
    const int kl = klg > 0 ? (int)nlo[r] : 0, ku = kug > 0 ? (int)nup[r] : 0;
    const T term = row_off<T>(n, KL, r, kl, ku, col, aoff, x);
    if (SOR) x[r] = w * (term + b[r]) / diag[r] + (T(1) - w) * x[r];
    else x[r] = (term + b[r]) / diag[r];
  }
}

// ----------------------------------------------------------------------------
// Diagonal incomplete Cholesky factor, one group (iccg.f90:62-66 with the
// 1e-3 pivot floor; iccgstab.f90:34-38 without it, plus 1e-20):
//   d_r = 1 / (diag_r - sum_{lower} d_j aoff_rj^2)
template <typename T, bool STAB>
__global__ void __launch_bounds__(TPB) k_dic(int n, int r0, int r1, int klg, const int* __restrict__ col,
                                             const signed char* __restrict__ nlo, const T* __restrict__ aoff,
                                             const T* __restrict__ diag, T* d) {
  for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
    const int kl = klg > 0 ? (int)nlo[r] : 0;
    T dr = diag[r];
#pragma unroll
    for (int s = 0; s < KMAX; ++s)
      if (s < kl) {
        const T a = aoff[(size_t)s * n + r];
        dr = dr - d[col[(size_t)s * n + r]] * (a * a);
      }
    d[r] = STAB ? T(1) / dr + T(1.0e-20) : T(1) / fmax(dr, T(1.0e-3));
  }
}

// Forward sweep of the factor, one group: z_r = (y_r + sum_{lower} aoff z_j) d_r.
template <typename T>
__global__ void __launch_bounds__(TPB) k_dic_fwd(int n, int r0, int r1, int klg, const int* __restrict__ col,
                                                 const signed char* __restrict__ nlo, const T* __restrict__ aoff,
                                                 const T* __restrict__ d, const T* __restrict__ y, T* z,
                                                 const DevState* st) {
  if (st->done) return;
  for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
    const int kl = klg > 0 ? (int)nlo[r] : 0;
    T acc = y[r];
#pragma unroll
    for (int s = 0; s < KMAX; ++s)
      if (s < kl) acc = acc + aoff[(size_t)s * n + r] * z[col[(size_t)s * n + r]];
    z[r] = acc * d[r];
  }
}

// Backward sweep, one group, with the division by the diagonal folded in:
//   z_r = (z_r / (d_r + eps) + sum_{upper} aoff z_k) d_r.
template <typename T>
__global__ void __launch_bounds__(TPB) k_dic_bwd(int n, int r0, int r1, int KL, int kug,
                                                 const int* __restrict__ col, const signed char* __restrict__ nup,
                                                 const T* __restrict__ aoff, const T* __restrict__ d, T* z, T eps,
                                                 const DevState* st) {
  if (st->done) return;
  for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
    const int ku = kug > 0 ? (int)nup[r] : 0;
    T acc = z[r] / (d[r] + eps);
#pragma unroll
    for (int s = 0; s < KMAX; ++s)
      if (s < ku) acc = acc + aoff[(size_t)(KL + s) * n + r] * z[col[(size_t)(KL + s) * n + r]];
    z[r] = acc * d[r];
  }
}

// ----------------------------------------------------------------------------
// SIP (sip.f90:2-174).  Compass data per device row: neighbour rows
// cmp[k*n + r] (k = 0 N, 1 E, 2 S, 3 W; -1 for a dummy) and the face
// coefficients cf[k*n + r] (dummy faces included: they enter the factor).

// cf[k*n + r] = acoef(k+1, perm[r]+1)
template <typename T>
__global__ void __launch_bounds__(TPB) k_sip_coef(int n, int nmf, const int* __restrict__ perm,
                                                  const T* __restrict__ acoef, T* cf) {
  for (int r = blockIdx.x * TPB + threadIdx.x; r < n; r += gridDim.x * TPB) {
    const size_t i = (size_t)perm[r];
#pragma unroll
    for (int k = 0; k < 4; ++k) cf[(size_t)k * n + r] = acoef[i * nmf + k];
  }
}

// cf[k*n + r] = face coefficient k of device row r in a [nmf][nD] device-row array
template <typename T>
__global__ void __launch_bounds__(TPB) k_sip_coef_dev(int n, int nD, const T* __restrict__ face, T* cf) {
  for (int r = blockIdx.x * TPB + threadIdx.x; r < n; r += gridDim.x * TPB) {
#pragma unroll
    for (int k = 0; k < 4; ++k) cf[(size_t)k * n + r] = face[(size_t)k * nD + r];
  }
}

template <typename T>
struct SipFactor {
  T *lw, *ls, *lpr, *un, *ue;
};

template <typename T>
__device__ __forceinline__ T at_or0(const T* v, int j) { return j >= 0 ? v[j] : T(0); }

// Factor rows of one group (sip.f90:38-54; alpha = 0.92).
template <typename T>
__global__ void __launch_bounds__(TPB) k_sip_factor(int n, int r0, int r1, const int* __restrict__ cmp,
                                                    const T* __restrict__ cf, const T* __restrict__ diag,
                                                    SipFactor<T> f, T alpha) {
  for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
    const int s = cmp[(size_t)2 * n + r], w = cmp[(size_t)3 * n + r];
    const T un_s = at_or0(f.un, s), ue_s = at_or0(f.ue, s), un_w = at_or0(f.un, w), ue_w = at_or0(f.ue, w);
    const T lw = -cf[(size_t)2 * n + r] / (T(1) + alpha * un_s);
    const T ls = -cf[(size_t)3 * n + r] / (T(1) + alpha * ue_w);
    const T term1 = alpha * lw * un_s;
    const T term2 = alpha * ls * ue_w;
    const T lpr = T(1) / (diag[r] + term1 + term2 - (ls * un_w + lw * ue_s));
    f.lw[r] = lw;
    f.ls[r] = ls;
    f.lpr[r] = lpr;
    f.un[r] = -(cf[(size_t)1 * n + r] + term1) * lpr;
    f.ue[r] = -(cf[(size_t)0 * n + r] + term2) * lpr;
  }
}

// Forward sweep, one group: v_r = lpr_r (res_r - lw_r v_S - ls_r v_W)  (sip.f90:85-86).
template <typename T>
__global__ void __launch_bounds__(TPB) k_sip_fwd(int n, int r0, int r1, const int* __restrict__ cmp, SipFactor<T> f,
                                                 const T* __restrict__ res, T* v, const DevState* st) {
  if (st->done) return;
  for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
    const int s = cmp[(size_t)2 * n + r], w = cmp[(size_t)3 * n + r];
    v[r] = f.lpr[r] * (res[r] - f.lw[r] * at_or0(v, s) - f.ls[r] * at_or0(v, w));
  }
}

// Backward sweep, one group: v_r -= ue_r v_N + un_r v_E  (sip.f90:98-99).
template <typename T>
__global__ void __launch_bounds__(TPB) k_sip_bwd(int n, int r0, int r1, const int* __restrict__ cmp, SipFactor<T> f,
                                                 T* v, const DevState* st) {
  if (st->done) return;
  for (int r = r0 + blockIdx.x * TPB + threadIdx.x; r < r1; r += gridDim.x * TPB) {
    const int nn = cmp[r], e = cmp[(size_t)1 * n + r];
    v[r] = v[r] - f.ue[r] * at_or0(v, nn) - f.un[r] * at_or0(v, e);
  }
}

// ----------------------------------------------------------------------------
// All-row kernels (group table) with a fused reduction and the scalar update.

enum LegMode : int {
  LEG_SIP_RES = 0,    // res = b + O x - diag x; resn = sqrt(sum res^2 / n); res0 at the first iteration;
                      // marks the stop (sip.f90:65-76,104-110) for the end of the iteration
  LEG_RES_L1 = 1,     // res = b + O x - diag x; res0 = sum |res|               (iccg.f90:53-58)
  LEG_RES_L1_COPY = 2 // as LEG_RES_L1, plus reso = res                          (iccgstab.f90:26-31,39-45)
};

template <typename T, int MODE>
__global__ void __launch_bounds__(TPB) k_leg_resid(int n, int KL, GroupTab tab, const int* __restrict__ col,
                                                   const signed char* __restrict__ nlo,
                                                   const signed char* __restrict__ nup, const T* __restrict__ aoff,
                                                   const T* __restrict__ diag, const T* __restrict__ b,
                                                   const T* __restrict__ x, T* __restrict__ res,
                                                   T* __restrict__ reso, int nitermin, double* partials,
                                                   DevState* st) {
  if (st->done) return;
  const int g = tab_group(tab, blockIdx.x);
  const int stride = (tab.blk[g + 1] - tab.blk[g]) * TPB;
  double v[1] = {0.0};
  for (int r = tab.start[g] + (blockIdx.x - tab.blk[g]) * TPB + threadIdx.x; r < tab.start[g + 1]; r += stride) {
    const int kl = tab.kl[g] > 0 ? (int)nlo[r] : 0, ku = tab.ku[g] > 0 ? (int)nup[r] : 0;
    const T rr = (b[r] + row_off<T>(n, KL, r, kl, ku, col, aoff, x)) - diag[r] * x[r];
    res[r] = rr;
    if (MODE == LEG_RES_L1_COPY) reso[r] = rr;
    v[0] += MODE == LEG_SIP_RES ? (double)rr * (double)rr : fabs((double)rr);
  }
  if (grid_sum(v, partials, &st->ticket[6])) {
    if (!isfinite(v[0])) {
      st->nonfinite = 1;
      st->done = 1;
      return;
    }
    if (MODE == LEG_SIP_RES) {
      const double resn = sqrt(v[0] / (double)n);
      if (st->iter == 0) st->s[S_RES0] = resn;
      const double rsm = resn / fmax(st->s[S_RES0], 1.0e-6);
      st->s[S_RELRES] = rsm;
      st->converged = (st->iter + 1 > nitermin && rsm < 1.0e-3) ? 1 : 0;
      st->stop = (st->converged || rsm > 10.0) ? 1 : 0;
    } else {
      st->s[S_RES0] = v[0];
    }
  }
}

// End of a SIP iteration: count it and apply the stop marked by k_leg_resid.
__global__ void k_leg_finish(DevState* st) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || st->done) return;
  st->iter += 1;
  if (st->stop || st->iter >= st->maxit) st->done = 1;
}

// Start of a solve: counters and the scalars of the recurrences.
__global__ void k_leg_start(DevState* st, int maxit) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st->done = maxit <= 0 ? 1 : 0;
  st->iter = 0;
  st->inner = 0;
  st->maxit = maxit;
  st->converged = 0;
  st->nonfinite = 0;
  st->stop = 0;
  st->s[S_BET0] = 1.0e20;  // iccg.f90:68 (s0); iccgstab beto = 1 is set by the ICCGSTAB start
  st->s[S_RELRES] = 0.0;
}

enum LegVec : int {
  LV_SIP_ADD = 0,    // x += v                                   (sip.f90:101-103)
  LV_ICCG_P = 1,     // p = z + beta p                           (iccg.f90:86-90)
  LV_STAB_P = 2,     // p = r + om (p - alf u)                   (iccgstab.f90:58-60)
  LV_STAB_X = 3      // x += gam z; r -= gam u                   (iccgstab.f90:76-79)
};

template <typename T, int MODE>
__global__ void __launch_bounds__(TPB) k_leg_vec(int n, T* __restrict__ x, T* __restrict__ r, T* __restrict__ p,
                                                 const T* __restrict__ z, const T* __restrict__ u,
                                                 const DevState* st) {
  if (st->done) return;
  const T beta = (T)st->s[S_GAM], om = (T)st->s[S_OMG], alf = (T)st->s[S_ALF], gam = (T)st->s[S_GAM];
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    if (MODE == LV_SIP_ADD) x[i] = x[i] + z[i];
    if (MODE == LV_ICCG_P) p[i] = z[i] + beta * p[i];
    if (MODE == LV_STAB_P) p[i] = r[i] + om * (p[i] - alf * u[i]);
    if (MODE == LV_STAB_X) {
      x[i] = x[i] + gam * z[i];
      r[i] = r[i] - gam * u[i];
    }
  }
}

enum LegDot : int {
  LD_ICCG_SK = 0,   // sk = r.z; beta = sk / max(s0, 1e-10)               (iccg.f90:80-85)
  LD_STAB_BET = 1   // bet = r.reso; om = bet gam / (alf beto + 1e-20)    (iccgstab.f90:50-56)
};

template <typename T, int MODE>
__global__ void __launch_bounds__(TPB) k_leg_dot(int n, const T* __restrict__ a, const T* __restrict__ b,
                                                 double* partials, DevState* st) {
  if (st->done) return;
  double v[1] = {0.0};
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) v[0] += (double)a[i] * (double)b[i];
  if (grid_sum(v, partials, &st->ticket[6])) {
    if (MODE == LD_ICCG_SK) {
      st->s[S_BET] = v[0];
      st->s[S_GAM] = v[0] / fmax(st->s[S_BET0], 1.0e-10);
    } else {
      st->s[S_OMG] = v[0] * st->s[S_GAM] / (st->s[S_ALF] * st->s[S_BET0] + 1.0e-20);
      st->s[S_BET] = v[0];
      st->s[S_BET0] = v[0];
    }
  }
}

enum LegSpmv : int {
  LS_ICCG = 0,    // y = A p; s2 = p.y; alpha = sk / max(s2, 1e-10)         (iccg.f90:92-101)
  LS_STAB_U = 1,  // u = A z; ukreso = u.reso; gam = bet / (ukreso + 1e-20)  (iccgstab.f90:67-75)
  LS_STAB_V = 2   // v = A z; alf = v.r / (v.v + 1e-20)                      (iccgstab.f90:90-101)
};

template <typename T, int MODE>
__global__ void __launch_bounds__(TPB) k_leg_spmv(int n, int KL, GroupTab tab, const int* __restrict__ col,
                                                  const signed char* __restrict__ nlo,
                                                  const signed char* __restrict__ nup, const T* __restrict__ aoff,
                                                  const T* __restrict__ diag, const T* __restrict__ z,
                                                  T* __restrict__ y, const T* __restrict__ d1, double* partials,
                                                  DevState* st) {
  if (st->done) return;
  constexpr int NS = MODE == LS_STAB_V ? 2 : 1;
  const int g = tab_group(tab, blockIdx.x);
  const int stride = (tab.blk[g + 1] - tab.blk[g]) * TPB;
  double v[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) v[q] = 0.0;
  for (int r = tab.start[g] + (blockIdx.x - tab.blk[g]) * TPB + threadIdx.x; r < tab.start[g + 1]; r += stride) {
    const int kl = tab.kl[g] > 0 ? (int)nlo[r] : 0, ku = tab.ku[g] > 0 ? (int)nup[r] : 0;
    const T yr = diag[r] * z[r] - row_off<T>(n, KL, r, kl, ku, col, aoff, z);
    y[r] = yr;
    v[0] += (double)yr * (double)d1[r];
    if (MODE == LS_STAB_V) v[NS - 1] += (double)yr * (double)yr;
  }
  if (grid_sum(v, partials, &st->ticket[6])) {
    if (MODE == LS_ICCG) st->s[S_ALF] = st->s[S_BET] / fmax(v[0], 1.0e-10);
    if (MODE == LS_STAB_U) st->s[S_GAM] = st->s[S_BET] / (v[0] + 1.0e-20);
    if (MODE == LS_STAB_V) st->s[S_ALF] = v[0] / (v[NS - 1] + 1.0e-20);
  }
}

// Solution/residual update with the L1 stopping test (iccg.f90:103-121,
// iccgstab.f90:103-113): x += alf p; r -= alf q; resm = sum|r| / max(res0, 1e-10).
// ICCG also stops when resm > 10 and needs more than nitermin iterations.
template <typename T, bool ICCG>
__global__ void __launch_bounds__(TPB) k_leg_update(int n, T* __restrict__ x, T* __restrict__ r,
                                                    const T* __restrict__ p, const T* __restrict__ q, int nitermin,
                                                    double* partials, DevState* st) {
  if (st->done) return;
  const T alf = (T)st->s[S_ALF];
  double v[1] = {0.0};
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    x[i] = x[i] + alf * p[i];
    const T ri = r[i] - alf * q[i];
    r[i] = ri;
    v[0] += fabs((double)ri);
  }
  if (grid_sum(v, partials, &st->ticket[6])) {
    st->iter += 1;
    if (!isfinite(v[0])) {
      st->nonfinite = 1;
      st->done = 1;
      return;
    }
    const double resm = v[0] / fmax(st->s[S_RES0], 1.0e-10);
    st->s[S_RELRES] = resm;
    if (ICCG) {
      st->s[S_BET0] = st->s[S_BET];  // s0 = sk
      if (st->iter > nitermin && resm < 1.0e-3) { st->converged = 1; st->done = 1; }
      else if (resm > 10.0) st->done = 1;
    } else if (resm < 1.0e-3) {
      st->converged = 1;
      st->done = 1;
    }
    if (st->iter >= st->maxit) st->done = 1;
  }
}

// ICCGSTAB start scalars: alf = beto = gam = 1 (iccgstab.f90:46-48).
__global__ void k_stab_start(DevState* st) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st->s[S_ALF] = 1.0;
  st->s[S_BET0] = 1.0;
  st->s[S_GAM] = 1.0;
}

// ----------------------------------------------------------------------------
// Pipelined passes, for orderings with many groups (the natural ordering's
// level sets, one launch each above).  One launch runs one pass, or many
// Gauss-Seidel passes, over all rows.  The work unit is a chunk of at most TPB
// rows of one group, claimed in order through a ticket (pass-major; a
// backward pass takes the chunks in reverse order).  A row waits until each
// coupling on the pass's new side (lower slots forward, upper slots backward)
// has completed this pass, and each coupling on the old side and the row
// itself the previous one (done[j] counts the passes row j completed),
// computes, and publishes its count with a release store.  A unit waits only on rows of units with
// earlier tickets, which blocks that are already running hold, so the
// pipeline always advances.  Every wait is bounded: one that runs out sets
// *err (the host reports a device error) and the row goes on with what it
// has, so that the launch drains.  Values written in the launch are read
// through L2 (ld.global.cg): L1 is not coherent across SMs.

struct PipeSched {
  const int* cstart;     // [nchunk + 1] first device row of each chunk
  int nchunk;
  unsigned int* done;    // [n] passes completed per row
  unsigned int* ticket;  // work-unit counter of the launch (zero at launch)
  int* err;              // [8] err[0]: a wait ran out; err[1..5]: where (pipe_ready)
  unsigned int spin_limit;  // polls before a wait gives up (kSpinLimit)
};

// Waits until every row js[q] (bit q of vmask set) has completed needs[q]
// passes (the arrays are indexed by compile-time positions): all the
// flags are read together (relaxed), then one acquire fence orders the data
// loads that follow.  The first wait that runs out records where: err[1..5] =
// row waiting, a row not ready, its need, the count seen, unit.
template <int M>
__device__ __forceinline__ bool pipe_ready(const PipeSched& ps, const int (&js)[M], const unsigned int (&needs)[M],
                                           unsigned int vmask, int r, int unit) {
  unsigned int spins = 0;
  for (;;) {
    int badj = -1;
    unsigned int seen = 0, badneed = 0;
#pragma unroll
    for (int q = 0; q < M; ++q)
      if ((vmask >> q) & 1u) {
        const unsigned int v = ld_relaxed(&ps.done[js[q]]);
        if (v < needs[q]) { badj = js[q]; badneed = needs[q]; seen = v; }
      }
    if (badj < 0) break;
    if (++spins > ps.spin_limit) {
      if (atomicCAS(ps.err, 0, 1) == 0) {
        ps.err[1] = r; ps.err[2] = badj; ps.err[3] = (int)badneed; ps.err[4] = (int)seen; ps.err[5] = unit;
      }
      fence_acquire();
      return false;
    }
    if ((spins & 1023u) == 0 && *(volatile int*)ps.err) break;
  }
  fence_acquire();
  return true;
}

// Claims the next unit for the block; -1 when none is left.
__device__ __forceinline__ int pipe_claim(const PipeSched& ps, int total) {
  __shared__ int s_unit;
  __syncthreads();
  if (threadIdx.x == 0) s_unit = (int)atomicAdd(ps.ticket, 1u);
  __syncthreads();
  const int t = s_unit;
  return t < total ? t : -1;
}

// npass Gauss-Seidel passes (sym: alternately forward and backward) in one
// launch; base = passes the rows completed before it.  units (forward passes
// only; nullptr: pass-major order) lists the work units as (pass, chunk) in
// wavefront order: chunk c of level L in pass h comes with the others of
// wave L + 2h, after every unit it waits on, so that consecutive passes
// overlap instead of following each other.
template <typename T, bool SOR>
__global__ void __launch_bounds__(TPB) k_gs_pipe(int n, int KL, const int* __restrict__ col,
                                                 const signed char* __restrict__ nlo,
                                                 const signed char* __restrict__ nup, const T* __restrict__ aoff,
                                                 const T* __restrict__ diag, const T* __restrict__ b, T* x, T w,
                                                 PipeSched ps, int npass, int sym, unsigned int base,
                                                 const int2* __restrict__ units) {
  const int total = npass * ps.nchunk;
  for (int t; (t = pipe_claim(ps, total)) >= 0;) {
    int h, c;
    if (units) {
      const int2 u = units[t];
      h = u.x; c = u.y;
    } else {
      h = t / ps.nchunk;
      const int c0 = t - h * ps.nchunk;
      c = (sym && (h & 1)) ? ps.nchunk - 1 - c0 : c0;
    }
    const bool bwd = sym && (h & 1);
    const int r = ps.cstart[c] + threadIdx.x;
    if (r >= ps.cstart[c + 1]) continue;
    const unsigned int mine = base + (unsigned int)h + 1u;
    const int kl = nlo[r], ku = nup[r];
    // positions: 0 the row itself, 1..KMAX lower slots, KMAX+1..2 KMAX upper
    int js[1 + 2 * KMAX];
    unsigned int needs[1 + 2 * KMAX];
    T av[2 * KMAX];
    // the row itself: where the direction turns, its neighbours alone do not
    // order it (a row with couplings on the old side only could otherwise
    // start this pass before finishing the last one)
    js[0] = r; needs[0] = mine - 1u;
    unsigned int vmask = 1u;
#pragma unroll
    for (int s = 0; s < KMAX; ++s) {
      const bool lo = s < kl, up = s < ku;
      js[1 + s] = lo ? __ldg(&col[(size_t)s * n + r]) : r;
      av[s] = lo ? __ldg(&aoff[(size_t)s * n + r]) : T(0);
      needs[1 + s] = bwd ? mine - 1u : mine;
      js[1 + KMAX + s] = up ? __ldg(&col[(size_t)(KL + s) * n + r]) : r;
      av[KMAX + s] = up ? __ldg(&aoff[(size_t)(KL + s) * n + r]) : T(0);
      needs[1 + KMAX + s] = bwd ? mine : mine - 1u;
      vmask |= (lo ? 1u << (1 + s) : 0u) | (up ? 1u << (1 + KMAX + s) : 0u);
    }
    pipe_ready(ps, js, needs, vmask, r, t);
    T term = T(0);
#pragma unroll
    for (int s = 0; s < KMAX; ++s)
      if (s < kl) term = term + av[s] * __ldcg(&x[js[1 + s]]);
#pragma unroll
    for (int s = 0; s < KMAX; ++s)
      if (s < ku) term = term + av[KMAX + s] * __ldcg(&x[js[1 + KMAX + s]]);
    const T br = __ldg(&b[r]), dr = __ldg(&diag[r]);
    if (SOR) x[r] = w * (term + br) / dr + (T(1) - w) * __ldcg(&x[r]);
    else x[r] = (term + br) / dr;
    st_release(&ps.done[r], mine);
  }
}

// The wait of the pipelined passes on rows that never complete (test of the
// bounded wait: every thread of one block waits on row j of a done array
// nobody writes, gives up after ps.spin_limit polls and records it).
__global__ void k_pipe_wait_probe(PipeSched ps, int j) {
  int js[1] = {j};
  unsigned int needs[1] = {1u};
  pipe_ready(ps, js, needs, 1u, (int)threadIdx.x, 0);
}

// One pipelined pass of a triangular recurrence: Op::row(r) reads only rows
// on the pass's new side (through L2) and rows of earlier launches.
template <class Op>
__global__ void __launch_bounds__(TPB) k_tri_pipe(Op op, int n, int KL, const int* __restrict__ col,
                                                  const signed char* __restrict__ nlo,
                                                  const signed char* __restrict__ nup, PipeSched ps, int bwd,
                                                  unsigned int epoch, const DevState* st) {
  if (st && st->done) return;  // every block sees the same flag (set by an earlier launch)
  for (int t; (t = pipe_claim(ps, ps.nchunk)) >= 0;) {
    const int c = bwd ? ps.nchunk - 1 - t : t;
    const int r = ps.cstart[c] + threadIdx.x;
    if (r >= ps.cstart[c + 1]) continue;
    int js[KMAX];
    unsigned int needs[KMAX];
    const int m = bwd ? nup[r] : nlo[r];
    const size_t off = bwd ? (size_t)KL * n : 0;
    unsigned int vmask = 0u;
#pragma unroll
    for (int s = 0; s < KMAX; ++s) {
      js[s] = s < m ? __ldg(&col[off + (size_t)s * n + r]) : r;
      needs[s] = epoch;
      vmask |= s < m ? 1u << s : 0u;
    }
    pipe_ready(ps, js, needs, vmask, r, t);
    op.row(r);
    st_release(&ps.done[r], epoch);
  }
}

template <typename T>
__device__ __forceinline__ T cg_or0(const T* v, int j) { return j >= 0 ? __ldcg(&v[j]) : T(0); }

// The recurrences of k_dic, k_dic_fwd, k_dic_bwd, k_sip_factor, k_sip_fwd and
// k_sip_bwd, one row each, for k_tri_pipe.
template <typename T, bool STAB>
struct OpDicFactor {
  int n; const int* col; const signed char* nlo; const T* aoff; const T* diag; T* d;
  __device__ void row(int r) const {
    const int kl = nlo[r];
    T dr = diag[r];
    for (int s = 0; s < kl; ++s) {
      const T a = aoff[(size_t)s * n + r];
      dr = dr - __ldcg(&d[col[(size_t)s * n + r]]) * (a * a);
    }
    d[r] = STAB ? T(1) / dr + T(1.0e-20) : T(1) / fmax(dr, T(1.0e-3));
  }
};

template <typename T>
struct OpDicFwd {
  int n; const int* col; const signed char* nlo; const T* aoff; const T* d; const T* y; T* z;
  __device__ void row(int r) const {
    const int kl = nlo[r];
    T acc = y[r];
    for (int s = 0; s < kl; ++s) acc = acc + aoff[(size_t)s * n + r] * __ldcg(&z[col[(size_t)s * n + r]]);
    z[r] = acc * d[r];
  }
};

template <typename T>
struct OpDicBwd {
  int n, KL; const int* col; const signed char* nup; const T* aoff; const T* d; T* z; T eps;
  __device__ void row(int r) const {
    const int ku = nup[r];
    T acc = __ldcg(&z[r]) / (d[r] + eps);
    for (int s = 0; s < ku; ++s)
      acc = acc + aoff[(size_t)(KL + s) * n + r] * __ldcg(&z[col[(size_t)(KL + s) * n + r]]);
    z[r] = acc * d[r];
  }
};

template <typename T>
struct OpSipFactor {
  int n; const int* cmp; const T* cf; const T* diag; SipFactor<T> f; T alpha;
  __device__ void row(int r) const {
    const int s = cmp[(size_t)2 * n + r], w = cmp[(size_t)3 * n + r];
    const T un_s = cg_or0(f.un, s), ue_s = cg_or0(f.ue, s), un_w = cg_or0(f.un, w), ue_w = cg_or0(f.ue, w);
    const T lw = -cf[(size_t)2 * n + r] / (T(1) + alpha * un_s);
    const T ls = -cf[(size_t)3 * n + r] / (T(1) + alpha * ue_w);
    const T term1 = alpha * lw * un_s;
    const T term2 = alpha * ls * ue_w;
    const T lpr = T(1) / (diag[r] + term1 + term2 - (ls * un_w + lw * ue_s));
    f.lw[r] = lw;
    f.ls[r] = ls;
    f.lpr[r] = lpr;
    f.un[r] = -(cf[(size_t)1 * n + r] + term1) * lpr;
    f.ue[r] = -(cf[(size_t)0 * n + r] + term2) * lpr;
  }
};

template <typename T>
struct OpSipFwd {
  int n; const int* cmp; SipFactor<T> f; const T* res; T* v;
  __device__ void row(int r) const {
    const int s = cmp[(size_t)2 * n + r], w = cmp[(size_t)3 * n + r];
    v[r] = f.lpr[r] * (res[r] - f.lw[r] * cg_or0(v, s) - f.ls[r] * cg_or0(v, w));
  }
};

template <typename T>
struct OpSipBwd {
  int n; const int* cmp; SipFactor<T> f; T* v;
  __device__ void row(int r) const {
    const int nn = cmp[r], e = cmp[(size_t)1 * n + r];
    v[r] = __ldcg(&v[r]) - f.ue[r] * cg_or0(v, nn) - f.un[r] * cg_or0(v, e);
  }
};

}  // namespace cms
