// Adjoint of solve() (included at the end of cms_solver.cu).
//
// solve() turns (acoef, ss, sp, phi) into A x = b with
//   A_ii = ap_i = (sum_k acoef(k,i) - sp_i) / relax,   A_ic = -acoef(k,i)  (c active),
//   b_i  = ss_i + (1 - relax) phi_i ap_i + sum_{k: c dummy} acoef(k,i) phi_c
// (solvers.f90:230-240).  For a loss L(x) with g = dL/dx the adjoint solve is
// A^T lam = g, and
//   dL/dss_i       = lam_i
//   dL/dsp_i       = lam_i (x_i - (1 - relax) phi_i) / relax
//   dL/dacoef(k,i) = lam_i ((1 - relax) phi_i - x_i) / relax + lam_i x_c
// where x_c is the solution at an active neighbour and phi_c at a dummy.
//
// A^T has A's sparsity pattern: its ELL values are A's entries read through a
// transpose map (slot e of row r holds the slot of row col[e] that points back
// to r).  It is solved by the same ILU(0)-BiCGStab (ILU(0) of A^T in the same
// device order), FP64.
#pragma once

namespace cms {

// aT[e] = a[tslot[e]] (0 where the slot is padding)
template <typename T>
__global__ void __launch_bounds__(TPB) k_transpose_vals(size_t m, const int* __restrict__ tslot,
                                                        const T* __restrict__ a, T* __restrict__ aT) {
  for (size_t e = (size_t)blockIdx.x * TPB + threadIdx.x; e < m; e += (size_t)gridDim.x * TPB) {
    const int t = tslot[e];
    aT[e] = t >= 0 ? a[t] : T(0);
  }
}

// b[r] = g[perm[r]] (natural -> device order)
__global__ void __launch_bounds__(TPB) k_gather_rhs(int n, const int* __restrict__ perm, const double* __restrict__ g,
                                                    double* __restrict__ b) {
  for (int r = blockIdx.x * TPB + threadIdx.x; r < n; r += gridDim.x * TPB) b[r] = g[perm[r]];
}

// gradients with respect to the solve() inputs, natural order (see above)
__global__ void __launch_bounds__(TPB) k_solve_grads(int n, int nmf, const int* __restrict__ c2c,
                                                     const int* __restrict__ ncface, const int* __restrict__ iperm,
                                                     const double* __restrict__ lam_dev,
                                                     const double* __restrict__ x, const double* __restrict__ phi0,
                                                     double relax, double* __restrict__ lam, double* __restrict__ gac,
                                                     double* __restrict__ gss, double* __restrict__ gsp) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    const double l = lam_dev[iperm[i]];
    const double xi = x[i];
    const double dap = l * ((1.0 - relax) * phi0[i] - xi) / relax;  // dL/d(acoef) through ap and b
    if (lam) lam[i] = l;
    if (gss) gss[i] = l;
    if (gsp) gsp[i] = -dap;
    if (gac) {
      const int nf = ncface[i];
      for (int k = 0; k < nmf; ++k) {
        double v = 0.0;
        if (k < nf) v = dap + l * x[c2c[(size_t)i * nmf + k] - 1];
        gac[(size_t)i * nmf + k] = v;
      }
    }
  }
}

// transpose map and buffers of A^T (first use)
static int adjoint_setup(Solver* S) {
  if (S->d_tslot) return CMS_OK;
  const HostPattern& P = S->hp;
  const size_t n = P.n, K = std::max(S->K, 1);
  std::vector<int> ts(K * n, -1);
  for (size_t r = 0; r < n; ++r) {
    const int kl = P.nlo[r], ku = P.nup[r];
    for (int s = 0; s < S->K; ++s) {
      const bool valid = s < P.KL ? s < kl : (s - P.KL) < ku;
      if (!valid) continue;
      const int j = P.col[(size_t)s * n + r];
      // row j's slot pointing back to r: an upper slot of j when j < r
      const int a0 = j < (int)r ? P.KL : 0, a1 = j < (int)r ? P.KL + P.nup[j] : P.nlo[j];
      for (int s2 = a0; s2 < a1; ++s2)
        if (P.col[(size_t)s2 * n + j] == (int)r) {
          ts[(size_t)s * n + r] = (int)((size_t)s2 * n + j);
          break;
        }
      if (ts[(size_t)s * n + r] < 0) {
        std::snprintf(g_last_error, sizeof(g_last_error), "adjoint: pattern is not symmetric at row %zu", r);
        return CMS_UNSUPPORTED;
      }
    }
  }
  int* d = nullptr;
  CHK(S->alloc(&d, K * n));
  CMS_CUDA(cudaMemcpyAsync(d, ts.data(), K * n * sizeof(int), cudaMemcpyHostToDevice, S->stream));
  CHK(S->alloc(&S->AT64.aoff, K * n));
  CHK(S->alloc(&S->AT64.luoff, K * n));
  CHK(S->alloc(&S->AT64.invd, n));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  S->d_tslot = d;
  return CMS_OK;
}

// A^T lam = g and the gradients of solve()'s inputs (all natural order,
// device pointers; see cms_solver_adjoint_dev_d).
static int solve_adjoint(Solver* S, const double* acoef, const double* ss, const double* sp, const double* phi0,
                         const double* x, double relax, const double* g, double tol, int maxit, double* lam,
                         double* gac, double* gss, double* gsp, cms_solve_info* info) {
  const HostPattern& P = S->hp;
  const int n = P.n;
  cms_solve_info loc{};
  if (!info) info = &loc;
  std::memset(info, 0, sizeof(*info));
  info->ncolors = P.G;
  info->true_relres = -1.0;
  CHK(adjoint_setup(S));
  CHK(alloc_staging<double>(S, S->S64));
  cudaStream_t st = S->stream;
  const size_t nD = P.nD, nmf = P.nmf;
  // the forward system again (ss on a copy: the prologue updates it in place)
  CMS_CUDA(cudaMemcpyAsync(S->S64.ss, ss, nD * sizeof(double), cudaMemcpyDeviceToDevice, st));
  KLAUNCH(S, P_PROLOGUE, 0.0,
          (k_prologue<double, float><<<gsz(n), TPB, 0, st>>>(n, (int)nmf, acoef, S->S64.ss, sp, S->S64.res, phi0,
                                                              S->d_c2c, S->d_ncface, S->d_iwet, S->d_fslot,
                                                              S->d_iperm, relax, S->A64.aoff, S->A64.diag,
                                                              S->W64.b, S->W64.x, nullptr, nullptr, S->d_part,
                                                              S->d_st)));
  const size_t m = (size_t)std::max(S->K, 1) * n;
  S->AT64.diag = S->A64.diag;
  KLAUNCH(S, P_VEC, (double)m * 20,
          (k_transpose_vals<double><<<gsz(n), TPB, 0, st>>>(m, S->d_tslot, S->A64.aoff, S->AT64.aoff)));
  KLAUNCH(S, P_VEC, (double)n * 20, (k_gather_rhs<<<gsz(n), TPB, 0, st>>>(n, S->d_perm, g, S->W64.b)));
  const int saved_relax = S->cur_relax;
  S->cur_relax = 0;
  CHK(run_bicgstab<double>(S, S->AT64, S->W64, maxit, 2, tol, 1, true));
  S->cur_relax = saved_relax;
  CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, st));
  CMS_CUDA(cudaStreamSynchronize(st));
  const DevState& h = *S->h_st;
  info->iters = h.iter;
  info->inner = h.iter;
  info->relres = h.s[S_RELRES];
  if (h.nonfinite) info->status = CMS_NONFINITE;
  else if (!h.converged) info->status = CMS_NOT_CONVERGED;
  KLAUNCH(S, P_VEC, (double)n * (8 * 6 + nmf * 20),
          (k_solve_grads<<<gsz(n), TPB, 0, st>>>(n, (int)nmf, S->d_c2c, S->d_ncface, S->d_iperm, S->W64.x, x, phi0,
                                                 relax, lam, gac, gss, gsp)));
  CMS_CUDA(cudaStreamSynchronize(st));
  return info->status;
}

// Bottom-friction sink of the momentum assembly and its adjoint.  Manning
// closure (fric_eval, friction.F90:647-662; fric_lib.f90:965-966) as the
// flow step evaluates it (kf_fric_vis):
//   Cd = g n^2 / hh^p,   hh = max(min(10, h), 0.1 n),   p = 0.3333,
// and the sink of coeffsourcesink_uv (flow_imp.F90:409-574, kf_coef_uv):
//   sp = spuv0 - Cd |u| A.
// With h, |u| and A held fixed, dsp/dn = -|u| A dCd/dn, where dCd/dn =
// 2 g n / hh^p on the depth branch and (2 - p) Cd / n where 0.1 n is the
// larger (a kink where the two meet; the depth branch is taken there).
constexpr double kManningP = 0.3333;

__device__ __forceinline__ double manning_cd(double g, double n, double h, double* dcd) {
  const double hd = fmin(10.0, h);
  const double hh = fmax(hd, 0.1 * n);
  const double cd = g * n * n / pow(hh, kManningP);
  if (dcd) *dcd = (0.1 * n > hd) ? (2.0 - kManningP) * cd / n : 2.0 * g * n / pow(hh, kManningP);
  return cd;
}

__global__ void __launch_bounds__(TPB) k_fric_sink(int n, double g, const double* __restrict__ coefman,
                                                   const double* __restrict__ h, const double* __restrict__ uv,
                                                   const double* __restrict__ area,
                                                   const double* __restrict__ spuv0, double* __restrict__ sp) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB)
    sp[i] = spuv0[i] - manning_cd(g, coefman[i], h[i], nullptr) * uv[i] * area[i];
}

__global__ void __launch_bounds__(TPB) k_fric_sink_adjoint(int n, double g, const double* __restrict__ coefman,
                                                           const double* __restrict__ h,
                                                           const double* __restrict__ uv,
                                                           const double* __restrict__ area,
                                                           const double* __restrict__ gsp,
                                                           double* __restrict__ gn) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    double dcd;
    manning_cd(g, coefman[i], h[i], &dcd);
    gn[i] = -gsp[i] * uv[i] * area[i] * dcd;
  }
}

// Momentum face coefficients of coeffsourcesink_uv (flow_imp.F90:409-574)
// and their adjoint: acoef(k,i) = scheme(D, F) with D = visk hk ds for the
// faces k < ncface(i) of the active cells, in the solve() layout
// ([ncellsD][nmaxfaces], natural order); the scheme is the flow step's own
// schemecoef (comp_lib.f90:40-109).  scheme_grad gives dA/dD and dA/dF of
// the branch the forward value takes (each function is piecewise smooth in
// (D, F); at a branch boundary the branch the comparisons below select).
__device__ __forceinline__ void scheme_grad(int ndsch, double dk, double fk, double& gD, double& gF) {
  const double absf = fabs(fk), sf = fk > 0.0 ? 1.0 : (fk < 0.0 ? -1.0 : 0.0);
  const double up = fk < 0.0 ? -1.0 : 0.0;  // d max(0, -F) / dF
  gD = 0.0;
  gF = 0.0;
  switch (ndsch) {
    case 0:
      return;
    case 2: {  // hybrid: D max(0, 1 - P/2), P = |F| / max(D, 1e-6)
      const double dp = fmax(dk, 1.0e-6), ddp = dk >= 1.0e-6 ? 1.0 : 0.0;
      const double pk = absf / dp, pD = -absf / (dp * dp) * ddp, pF = sf / dp;
      const double gg = 1.0 - 0.5 * pk;
      if (gg > 0.0) {
        gD = gg - 0.5 * dk * pD;
        gF = -0.5 * dk * pF;
      }
      gF += up;
      return;
    }
    case 3: {  // power law: D (1 - P^5), P = |F| / max(max(D, |F|), 1e-6)
      const double mm = fmax(dk, absf);
      const double m = fmax(mm, 1.0e-6);
      double mD = 0.0, mF = 0.0;
      if (mm >= 1.0e-6) {
        if (dk >= absf) mD = 1.0;
        else mF = sf;
      }
      const double pk = absf / m, pD = -absf / (m * m) * mD, pF = sf / m - absf / (m * m) * mF;
      const double p4 = pk * pk * pk * pk;
      gD = (1.0 - p4 * pk) - 5.0 * dk * p4 * pD;
      gF = -5.0 * dk * p4 * pF + up;
      return;
    }
    case 4: {  // exponential: D P / max(e^P - 1, 1e-6), P = |F| / max(max(D, 1e-6), |F|)
      const double dp = fmax(dk, 1.0e-6);
      const double m = fmax(dp, absf);
      const double mD = (dk >= 1.0e-6 && dp >= absf) ? 1.0 : 0.0, mF = absf > dp ? sf : 0.0;
      const double pk = absf / m, pD = -absf / (m * m) * mD, pF = sf / m - absf / (m * m) * mF;
      const double ex = exp(pk), e = fmax(ex - 1.0, 1.0e-6), eP = (ex - 1.0 > 1.0e-6) ? ex : 0.0;
      gD = pk / e + dk * pD / e - dk * pk * eP * pD / (e * e);
      gF = dk * pF / e - dk * pk * eP * pF / (e * e) + up;
      return;
    }
    default:  // upwind: D + max(0, -F)
      gD = 1.0;
      gF = up;
      return;
  }
}

__global__ void __launch_bounds__(TPB) k_mom_coef(int n, int nmf, int ndsch, const int* __restrict__ ncface,
                                                  const double* __restrict__ visk, const double* __restrict__ hk,
                                                  const double* __restrict__ ds, const double* __restrict__ flux,
                                                  double* __restrict__ acoef) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    const int nf = ncface[i];
    for (int k = 0; k < nf; ++k) {
      const size_t f = (size_t)i * nmf + k;
      acoef[f] = schemecoef(ndsch, visk[f] * hk[f] * ds[f], flux[f]);
    }
  }
}

__global__ void __launch_bounds__(TPB) k_mom_coef_adjoint(int n, int nmf, int ndsch, const int* __restrict__ ncface,
                                                          const double* __restrict__ visk,
                                                          const double* __restrict__ hk,
                                                          const double* __restrict__ ds,
                                                          const double* __restrict__ flux,
                                                          const double* __restrict__ ga, double* __restrict__ gvisk,
                                                          double* __restrict__ ghk, double* __restrict__ gflux) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    const int nf = ncface[i];
    for (int k = 0; k < nmf; ++k) {
      const size_t f = (size_t)i * nmf + k;
      double gD = 0.0, gF = 0.0;
      if (k < nf) scheme_grad(ndsch, visk[f] * hk[f] * ds[f], flux[f], gD, gF);
      const double g = ga[f];
      if (gvisk) gvisk[f] = g * gD * hk[f] * ds[f];
      if (ghk) ghk[f] = g * gD * visk[f] * ds[f];
      if (gflux) gflux[f] = g * gF;
    }
  }
}

// Pressure-correction coefficients of coefsourcesink_pp (flow_imp.F90:577-794,
// the flow step's kf_pp_cell / kf_pp_face without skewness correction) from the
// momentum coefficients, and their adjoint.  Per active cell
//   Dn = sum_k acoef_u(k,i) - sp_u(i),  apu = iwet relax / max(Dn, 1e-6),
//   ap = apu A,  sumu = (sum_k acoef_u) apu,
// per face k < ncface(i) to a wet cell c (else 0):
//   a_pp = hk^2 ds ap_f / (1 - sumu_f) / dn,
// with ap_f, sumu_f the cell values for a dummy neighbour and
// fintp ap(c) + (1 - fintp) ap(i) (the same for sumu) for an active one.
// Face fields in the solve() layout ([ncellsD][nmaxfaces], 1-based cell2cell);
// fintp(kb, c) = 1 - fintp(k, i) on the two sides of a face keeps a_pp
// symmetric, as the flow step's mirrored faces.
struct PPCell {
  double ap, sumu, asum, dn;
};
__device__ __forceinline__ PPCell pp_cell(int i, int nmf, const int* ncface, const int* iwet, double relax,
                                          const double* acoef_u, const double* sp_u, const double* area) {
  PPCell c;
  c.asum = 0.0;
  for (int k = 0; k < ncface[i]; ++k) c.asum += acoef_u[(size_t)i * nmf + k];
  c.dn = c.asum - sp_u[i];
  const double apu = iwet[i] * relax / fmax(c.dn, 1.0e-6);
  c.ap = apu * area[i];
  c.sumu = c.asum * apu;
  return c;
}

__global__ void __launch_bounds__(TPB) k_pp_coef(int n, int nmf, const int* __restrict__ c2c,
                                                 const int* __restrict__ ncface, const int* __restrict__ iwet,
                                                 double relax, const double* __restrict__ acoef_u,
                                                 const double* __restrict__ sp_u, const double* __restrict__ area,
                                                 const double* __restrict__ hk, const double* __restrict__ ds,
                                                 const double* __restrict__ dn, const double* __restrict__ fintp,
                                                 double* __restrict__ acoef_pp) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    const PPCell ci = pp_cell(i, nmf, ncface, iwet, relax, acoef_u, sp_u, area);
    for (int k = 0; k < ncface[i]; ++k) {
      const size_t f = (size_t)i * nmf + k;
      const int c = c2c[f] - 1;
      double a = 0.0;
      if (iwet[i] * iwet[c] != 0) {
        const double K = hk[f] * hk[f] * ds[f] / dn[f];
        if (c >= n) {
          a = K * ci.ap / (1.0 - ci.sumu);
        } else {
          const PPCell cc = pp_cell(c, nmf, ncface, iwet, relax, acoef_u, sp_u, area);
          const double fk = fintp[f];
          a = K * (fk * cc.ap + (1.0 - fk) * ci.ap) / (1.0 - (fk * cc.sumu + (1.0 - fk) * ci.sumu));
        }
      }
      acoef_pp[f] = a;
    }
  }
}

// The adjoint as a gather: cell j collects dL/dap(j) and dL/dsumu(j) from its
// own faces (weight 1 - fintp, or 1 for a dummy neighbour) and from the faces
// of its neighbours that point back to it (weight their fintp), then turns
// them into dL/dacoef_u(., j) (one value for the row's faces) and dL/dsp_u(j);
// dL/dhk from the face's own coefficient.
__global__ void __launch_bounds__(TPB) k_pp_coef_adjoint(int n, int nmf, const int* __restrict__ c2c,
                                                         const int* __restrict__ ncface,
                                                         const int* __restrict__ iwet, double relax,
                                                         const double* __restrict__ acoef_u,
                                                         const double* __restrict__ sp_u,
                                                         const double* __restrict__ area,
                                                         const double* __restrict__ hk,
                                                         const double* __restrict__ ds,
                                                         const double* __restrict__ dn,
                                                         const double* __restrict__ fintp,
                                                         const double* __restrict__ ga, double* __restrict__ gacoef_u,
                                                         double* __restrict__ gsp_u, double* __restrict__ ghk) {
  for (int j = blockIdx.x * TPB + threadIdx.x; j < n; j += gridDim.x * TPB) {
    const PPCell cj = pp_cell(j, nmf, ncface, iwet, relax, acoef_u, sp_u, area);
    double gap = 0.0, gsu = 0.0;
    const int nfj = ncface[j];
    for (int k = 0; k < nmf; ++k) {
      const size_t f = (size_t)j * nmf + k;
      double gh = 0.0;
      const int c = k < nfj ? c2c[f] - 1 : -1;
      if (c >= 0 && iwet[j] * iwet[c] != 0) {
        const double K = hk[f] * hk[f] * ds[f] / dn[f], dK = 2.0 * hk[f] * ds[f] / dn[f];
        if (c >= n) {
          const double den = 1.0 - cj.sumu;
          gap += ga[f] * K / den;
          gsu += ga[f] * K * cj.ap / (den * den);
          gh = ga[f] * dK * cj.ap / den;
        } else {
          const PPCell cc = pp_cell(c, nmf, ncface, iwet, relax, acoef_u, sp_u, area);
          const double fk = fintp[f];
          const double apv = fk * cc.ap + (1.0 - fk) * cj.ap, den = 1.0 - (fk * cc.sumu + (1.0 - fk) * cj.sumu);
          gap += ga[f] * K / den * (1.0 - fk);
          gsu += ga[f] * K * apv / (den * den) * (1.0 - fk);
          gh = ga[f] * dK * apv / den;
          // the neighbour's faces that point back to j
          for (int kb = 0; kb < ncface[c]; ++kb) {
            const size_t fb = (size_t)c * nmf + kb;
            if (c2c[fb] - 1 != j) continue;
            const double Kb = hk[fb] * hk[fb] * ds[fb] / dn[fb], fkb = fintp[fb];
            const double apb = fkb * cj.ap + (1.0 - fkb) * cc.ap;
            const double denb = 1.0 - (fkb * cj.sumu + (1.0 - fkb) * cc.sumu);
            gap += ga[fb] * Kb / denb * fkb;
            gsu += ga[fb] * Kb * apb / (denb * denb) * fkb;
          }
        }
      }
      if (ghk) ghk[f] = gh;
    }
    // ap = w r A / max(Dn, 1e-6), sumu = asum w r / max(Dn, 1e-6), Dn = asum - sp
    const double w = iwet[j] * relax;
    double gasum, gsp;
    if (cj.dn > 1.0e-6) {
      const double d2 = cj.dn * cj.dn;
      gasum = gap * (-w * area[j] / d2) + gsu * (w * (-sp_u[j]) / d2);
      gsp = gap * (w * area[j] / d2) + gsu * (w * cj.asum / d2);
    } else {
      gasum = gsu * w / 1.0e-6;
      gsp = 0.0;
    }
    if (gacoef_u)
      for (int k = 0; k < nmf; ++k) gacoef_u[(size_t)j * nmf + k] = k < nfj ? gasum : 0.0;
    if (gsp_u) gsp_u[j] = gsp;
  }
}

// Right-hand side of the pressure-correction system (coefsourcesink_pp and
// the Rhie-Chow fluxes of flow_imp_flux_noskew, flow_imp_flux.f90:361-409,
// as the flow step's kf_pp_face / kf_pp_src evaluate them on wet cells
// without skewness correction), and its adjoint with respect to the momentum
// system (through apuareap) and the face depth:
//   Hu = u + ap dpx h,  Hv = v + ap dpy h,
//   flux(k,i) = hk ds (nx Hu_f + ny Hv_f - ap_f hk (p_c - p_i) / dn)
// (outward normal of face k of cell i from its direction 1 N, 2 E, 3 S, 4 W;
// face values interpolated with fintp, the cell's own at a dummy neighbour;
// 0 across a dry side), ss_pp(i) = sspp0(i) - sum_k flux(k,i) + p(i) sppp0(i).
__device__ __forceinline__ double pp_face_flux(int i, int k, int n, int nmf, const int* c2c, const int* idir,
                                               const int* iwet, const double* u, const double* v, const double* h,
                                               const double* dpx, const double* dpy, const double* p,
                                               const double* hk, const double* ds, const double* dn,
                                               const double* fintp, double api, double apc) {
  const size_t f = (size_t)i * nmf + k;
  const int c = c2c[f] - 1;
  if (iwet[i] * iwet[c] == 0) return 0.0;
  const double nx = fnxd(idir[f]), ny = fnyd(idir[f]);
  const double hui = u[i] + api * dpx[i] * h[i], hvi = v[i] + api * dpy[i] * h[i];
  double huf = hui, hvf = hvi, apf = api;
  if (c < n) {
    const double fk = fintp[f];
    huf = fk * (u[c] + apc * dpx[c] * h[c]) + (1.0 - fk) * hui;
    hvf = fk * (v[c] + apc * dpy[c] * h[c]) + (1.0 - fk) * hvi;
    apf = fk * apc + (1.0 - fk) * api;
  }
  return hk[f] * ds[f] * (nx * huf + ny * hvf - apf * hk[f] * (p[c] - p[i]) / dn[f]);
}

__global__ void __launch_bounds__(TPB) k_pp_rhs(int n, int nmf, const int* __restrict__ c2c,
                                                const int* __restrict__ ncface, const int* __restrict__ idir,
                                                const int* __restrict__ iwet, double relax,
                                                const double* __restrict__ acoef_u, const double* __restrict__ sp_u,
                                                const double* __restrict__ area, const double* __restrict__ u,
                                                const double* __restrict__ v, const double* __restrict__ h,
                                                const double* __restrict__ dpx, const double* __restrict__ dpy,
                                                const double* __restrict__ p, const double* __restrict__ hk,
                                                const double* __restrict__ ds, const double* __restrict__ dn,
                                                const double* __restrict__ fintp, const double* __restrict__ sspp0,
                                                const double* __restrict__ sppp0, double* __restrict__ ss_pp) {
  for (int i = blockIdx.x * TPB + threadIdx.x; i < n; i += gridDim.x * TPB) {
    const double api = pp_cell(i, nmf, ncface, iwet, relax, acoef_u, sp_u, area).ap;
    double sf = 0.0;
    for (int k = 0; k < ncface[i]; ++k) {
      const int c = c2c[(size_t)i * nmf + k] - 1;
      const double apc = c < n ? pp_cell(c, nmf, ncface, iwet, relax, acoef_u, sp_u, area).ap : 0.0;
      sf += pp_face_flux(i, k, n, nmf, c2c, idir, iwet, u, v, h, dpx, dpy, p, hk, ds, dn, fintp, api, apc);
    }
    ss_pp[i] = sspp0[i] - sf + p[i] * sppp0[i];
  }
}

// dflux(k,i)/dap(j) for j = i (own side, weight 1 - fintp, 1 at a dummy) or
// j = c (weight fintp), and dflux/dhk.
__device__ __forceinline__ void pp_flux_grads(int i, int k, int n, int nmf, const int* c2c, const int* idir,
                                              const int* iwet, const double* u, const double* v, const double* h,
                                              const double* dpx, const double* dpy, const double* p,
                                              const double* hk, const double* ds, const double* dn,
                                              const double* fintp, double api, double apc, double& d_api,
                                              double& d_apc, double& d_hk) {
  const size_t f = (size_t)i * nmf + k;
  const int c = c2c[f] - 1;
  d_api = d_apc = d_hk = 0.0;
  if (iwet[i] * iwet[c] == 0) return;
  const double nx = fnxd(idir[f]), ny = fnyd(idir[f]);
  const double K1 = hk[f] * ds[f], dp = (p[c] - p[i]) / dn[f];
  const double hui = u[i] + api * dpx[i] * h[i], hvi = v[i] + api * dpy[i] * h[i];
  if (c >= n) {
    d_api = K1 * (nx * dpx[i] * h[i] + ny * dpy[i] * h[i] - hk[f] * dp);
    d_hk = ds[f] * (nx * hui + ny * hvi) - 2.0 * hk[f] * ds[f] * api * dp;
    return;
  }
  const double fk = fintp[f], fp = 1.0 - fk;
  const double huc = u[c] + apc * dpx[c] * h[c], hvc = v[c] + apc * dpy[c] * h[c];
  const double huf = fk * huc + fp * hui, hvf = fk * hvc + fp * hvi, apf = fk * apc + fp * api;
  d_api = K1 * fp * (nx * dpx[i] * h[i] + ny * dpy[i] * h[i] - hk[f] * dp);
  d_apc = K1 * fk * (nx * dpx[c] * h[c] + ny * dpy[c] * h[c] - hk[f] * dp);
  d_hk = ds[f] * (nx * huf + ny * hvf) - 2.0 * hk[f] * ds[f] * apf * dp;
}

__global__ void __launch_bounds__(TPB) k_pp_rhs_adjoint(
    int n, int nmf, const int* __restrict__ c2c, const int* __restrict__ ncface, const int* __restrict__ idir,
    const int* __restrict__ iwet, double relax, const double* __restrict__ acoef_u, const double* __restrict__ sp_u,
    const double* __restrict__ area, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ h, const double* __restrict__ dpx, const double* __restrict__ dpy,
    const double* __restrict__ p, const double* __restrict__ hk, const double* __restrict__ ds,
    const double* __restrict__ dn, const double* __restrict__ fintp, const double* __restrict__ gss,
    double* __restrict__ gacoef_u, double* __restrict__ gsp_u, double* __restrict__ ghk, double* __restrict__ gu,
    double* __restrict__ gv) {
  for (int j = blockIdx.x * TPB + threadIdx.x; j < n; j += gridDim.x * TPB) {
    const PPCell cj = pp_cell(j, nmf, ncface, iwet, relax, acoef_u, sp_u, area);
    double gap = 0.0, guj = 0.0, gvj = 0.0;
    const int nfj = ncface[j];
    for (int k = 0; k < nmf; ++k) {
      const size_t f = (size_t)j * nmf + k;
      double gh = 0.0;
      if (k < nfj) {
        const int c = c2c[f] - 1;
        const double apc = c < n ? pp_cell(c, nmf, ncface, iwet, relax, acoef_u, sp_u, area).ap : 0.0;
        double da_i, da_c, dh;
        pp_flux_grads(j, k, n, nmf, c2c, idir, iwet, u, v, h, dpx, dpy, p, hk, ds, dn, fintp, cj.ap, apc, da_i,
                      da_c, dh);
        gap += -gss[j] * da_i;  // ss_pp(j) holds -flux(k,j)
        gh = -gss[j] * dh;
        if (iwet[j] * iwet[c] != 0) {  // dflux/du(j) = hk ds nx (j's interpolation weight)
          const double wj = (c < n ? 1.0 - fintp[f] : 1.0) * hk[f] * ds[f];
          guj += -gss[j] * wj * fnxd(idir[f]);
          gvj += -gss[j] * wj * fnyd(idir[f]);
        }
        if (c < n) {  // the neighbour's faces that point back to j: their flux depends on ap(j), u(j), v(j) too
          for (int kb = 0; kb < ncface[c]; ++kb) {
            const size_t fb = (size_t)c * nmf + kb;
            if (c2c[fb] - 1 != j) continue;
            double db_c, db_j, dhb;
            pp_flux_grads(c, kb, n, nmf, c2c, idir, iwet, u, v, h, dpx, dpy, p, hk, ds, dn, fintp, apc, cj.ap,
                          db_c, db_j, dhb);
            gap += -gss[c] * db_j;
            if (iwet[j] * iwet[c] != 0) {
              const double wb = fintp[fb] * hk[fb] * ds[fb];
              guj += -gss[c] * wb * fnxd(idir[fb]);
              gvj += -gss[c] * wb * fnyd(idir[fb]);
            }
          }
        }
      }
      if (ghk) ghk[f] = gh;
    }
    const double w = iwet[j] * relax;
    double gasum = 0.0, gsp = 0.0;
    if (cj.dn > 1.0e-6) {
      const double d2 = cj.dn * cj.dn;
      gasum = gap * (-w * area[j] / d2);
      gsp = gap * (w * area[j] / d2);
    }
    if (gacoef_u)
      for (int k = 0; k < nmf; ++k) gacoef_u[(size_t)j * nmf + k] = k < nfj ? gasum : 0.0;
    if (gsp_u) gsp_u[j] = gsp;
    if (gu) gu[j] = guj;
    if (gv) gv[j] = gvj;
  }
}

static int fric_launch_check(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) return CMS_OK;
  std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what, cudaGetErrorString(e));
  return CMS_DEVICE_ERROR;
}

}  // namespace cms

extern "C" int cms_fric_sink_dev_d(int n, double grav, const double* coefman, const double* h, const double* uv,
                                   const double* area, const double* spuv0, double* sp, void* stream) {
  if (n <= 0 || !coefman || !h || !uv || !area || !spuv0 || !sp) return CMS_BAD_ARGUMENT;
  const int blocks = std::max(1, std::min((n + cms::TPB - 1) / cms::TPB, 148 * 8));
  cms::k_fric_sink<<<blocks, cms::TPB, 0, (cudaStream_t)stream>>>(n, grav, coefman, h, uv, area, spuv0, sp);
  return cms::fric_launch_check("cms_fric_sink_dev_d");
}

extern "C" int cms_fric_sink_adjoint_dev_d(int n, double grav, const double* coefman, const double* h,
                                           const double* uv, const double* area, const double* grad_sp,
                                           double* grad_coefman, void* stream) {
  if (n <= 0 || !coefman || !h || !uv || !area || !grad_sp || !grad_coefman) return CMS_BAD_ARGUMENT;
  const int blocks = std::max(1, std::min((n + cms::TPB - 1) / cms::TPB, 148 * 8));
  cms::k_fric_sink_adjoint<<<blocks, cms::TPB, 0, (cudaStream_t)stream>>>(n, grav, coefman, h, uv, area, grad_sp,
                                                                          grad_coefman);
  return cms::fric_launch_check("cms_fric_sink_adjoint_dev_d");
}

extern "C" int cms_momentum_coef_dev_d(int ncells, int nmaxfaces, int ndsch, const int* ncface, const double* visk,
                                       const double* hk, const double* ds, const double* flux, double* acoef,
                                       void* stream) {
  if (ncells <= 0 || nmaxfaces <= 0 || nmaxfaces > 8 || ndsch < 0 || ndsch > 4 || !ncface || !visk || !hk || !ds ||
      !flux || !acoef)
    return CMS_BAD_ARGUMENT;
  const int blocks = std::max(1, std::min((ncells + cms::TPB - 1) / cms::TPB, 148 * 8));
  cms::k_mom_coef<<<blocks, cms::TPB, 0, (cudaStream_t)stream>>>(ncells, nmaxfaces, ndsch, ncface, visk, hk, ds,
                                                                 flux, acoef);
  return cms::fric_launch_check("cms_momentum_coef_dev_d");
}

extern "C" int cms_momentum_coef_adjoint_dev_d(int ncells, int nmaxfaces, int ndsch, const int* ncface,
                                               const double* visk, const double* hk, const double* ds,
                                               const double* flux, const double* grad_acoef, double* grad_visk,
                                               double* grad_hk, double* grad_flux, void* stream) {
  if (ncells <= 0 || nmaxfaces <= 0 || nmaxfaces > 8 || ndsch < 0 || ndsch > 4 || !ncface || !visk || !hk || !ds ||
      !flux || !grad_acoef)
    return CMS_BAD_ARGUMENT;
  const int blocks = std::max(1, std::min((ncells + cms::TPB - 1) / cms::TPB, 148 * 8));
  cms::k_mom_coef_adjoint<<<blocks, cms::TPB, 0, (cudaStream_t)stream>>>(ncells, nmaxfaces, ndsch, ncface, visk, hk,
                                                                         ds, flux, grad_acoef, grad_visk, grad_hk,
                                                                         grad_flux);
  return cms::fric_launch_check("cms_momentum_coef_adjoint_dev_d");
}

extern "C" int cms_pp_coef_dev_d(int ncells, int nmaxfaces, const int* cell2cell, const int* ncface, const int* iwet,
                                 double relax, const double* acoef_u, const double* sp_u, const double* area,
                                 const double* hk, const double* ds, const double* dn, const double* fintp,
                                 double* acoef_pp, void* stream) {
  if (ncells <= 0 || nmaxfaces <= 0 || nmaxfaces > 8 || relax <= 0.0 || !cell2cell || !ncface || !iwet ||
      !acoef_u || !sp_u || !area || !hk || !ds || !dn || !fintp || !acoef_pp)
    return CMS_BAD_ARGUMENT;
  const int blocks = std::max(1, std::min((ncells + cms::TPB - 1) / cms::TPB, 148 * 8));
  cms::k_pp_coef<<<blocks, cms::TPB, 0, (cudaStream_t)stream>>>(ncells, nmaxfaces, cell2cell, ncface, iwet, relax,
                                                                acoef_u, sp_u, area, hk, ds, dn, fintp, acoef_pp);
  return cms::fric_launch_check("cms_pp_coef_dev_d");
}

extern "C" int cms_pp_coef_adjoint_dev_d(int ncells, int nmaxfaces, const int* cell2cell, const int* ncface,
                                         const int* iwet, double relax, const double* acoef_u, const double* sp_u,
                                         const double* area, const double* hk, const double* ds, const double* dn,
                                         const double* fintp, const double* grad_acoef_pp, double* grad_acoef_u,
                                         double* grad_sp_u, double* grad_hk, void* stream) {
  if (ncells <= 0 || nmaxfaces <= 0 || nmaxfaces > 8 || relax <= 0.0 || !cell2cell || !ncface || !iwet ||
      !acoef_u || !sp_u || !area || !hk || !ds || !dn || !fintp || !grad_acoef_pp)
    return CMS_BAD_ARGUMENT;
  const int blocks = std::max(1, std::min((ncells + cms::TPB - 1) / cms::TPB, 148 * 8));
  cms::k_pp_coef_adjoint<<<blocks, cms::TPB, 0, (cudaStream_t)stream>>>(ncells, nmaxfaces, cell2cell, ncface, iwet,
                                                                        relax, acoef_u, sp_u, area, hk, ds, dn,
                                                                        fintp, grad_acoef_pp, grad_acoef_u, grad_sp_u,
                                                                        grad_hk);
  return cms::fric_launch_check("cms_pp_coef_adjoint_dev_d");
}

extern "C" int cms_pp_rhs_dev_d(int ncells, int nmaxfaces, const int* cell2cell, const int* ncface, const int* idirface,
                                const int* iwet, double relax, const double* acoef_u, const double* sp_u,
                                const double* area, const double* u, const double* v, const double* h,
                                const double* dpx, const double* dpy, const double* p, const double* hk,
                                const double* ds, const double* dn, const double* fintp, const double* sspp0,
                                const double* sppp0, double* ss_pp, void* stream) {
  if (ncells <= 0 || nmaxfaces <= 0 || nmaxfaces > 8 || relax <= 0.0 || !cell2cell || !ncface || !idirface ||
      !iwet || !acoef_u || !sp_u || !area || !u || !v || !h || !dpx || !dpy || !p || !hk || !ds || !dn || !fintp ||
      !sspp0 || !sppp0 || !ss_pp)
    return CMS_BAD_ARGUMENT;
  const int blocks = std::max(1, std::min((ncells + cms::TPB - 1) / cms::TPB, 148 * 8));
  cms::k_pp_rhs<<<blocks, cms::TPB, 0, (cudaStream_t)stream>>>(ncells, nmaxfaces, cell2cell, ncface, idirface, iwet,
                                                               relax, acoef_u, sp_u, area, u, v, h, dpx, dpy, p, hk,
                                                               ds, dn, fintp, sspp0, sppp0, ss_pp);
  return cms::fric_launch_check("cms_pp_rhs_dev_d");
}

extern "C" int cms_pp_rhs_adjoint_dev_d(int ncells, int nmaxfaces, const int* cell2cell, const int* ncface,
                                        const int* idirface, const int* iwet, double relax, const double* acoef_u,
                                        const double* sp_u, const double* area, const double* u, const double* v,
                                        const double* h, const double* dpx, const double* dpy, const double* p,
                                        const double* hk, const double* ds, const double* dn, const double* fintp,
                                        const double* grad_ss_pp, double* grad_acoef_u, double* grad_sp_u,
                                        double* grad_hk, double* grad_u, double* grad_v, void* stream) {
  if (ncells <= 0 || nmaxfaces <= 0 || nmaxfaces > 8 || relax <= 0.0 || !cell2cell || !ncface || !idirface ||
      !iwet || !acoef_u || !sp_u || !area || !u || !v || !h || !dpx || !dpy || !p || !hk || !ds || !dn || !fintp ||
      !grad_ss_pp)
    return CMS_BAD_ARGUMENT;
  const int blocks = std::max(1, std::min((ncells + cms::TPB - 1) / cms::TPB, 148 * 8));
  cms::k_pp_rhs_adjoint<<<blocks, cms::TPB, 0, (cudaStream_t)stream>>>(
      ncells, nmaxfaces, cell2cell, ncface, idirface, iwet, relax, acoef_u, sp_u, area, u, v, h, dpx, dpy, p, hk, ds,
      dn, fintp, grad_ss_pp, grad_acoef_u, grad_sp_u, grad_hk, grad_u, grad_v);
  return cms::fric_launch_check("cms_pp_rhs_adjoint_dev_d");
}

extern "C" int cms_solver_adjoint_dev_d(cms_solver* s, const double* acoef, const double* ss, const double* sp,
                                        const double* phi0, const double* x, double relax, const double* g,
                                        double tol, int maxit, double* lam, double* grad_acoef, double* grad_ss,
                                        double* grad_sp, cms_solve_info* info) {
  if (!s || !acoef || !ss || !sp || !phi0 || !x || !g || relax <= 0.0 || tol <= 0.0 || maxit <= 0)
    return CMS_BAD_ARGUMENT;
  return cms::solve_adjoint(s, acoef, ss, sp, phi0, x, relax, g, tol, maxit, lam, grad_acoef, grad_ss, grad_sp,
                            info);
}
