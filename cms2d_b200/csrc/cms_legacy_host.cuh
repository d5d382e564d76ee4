// Host drivers of the MATRIX_SOLVER options other than BiCGStab and GMRES
// (source/solvers/solvers.f90:242-289); kernels in cms_legacy.cuh.  Included
// by cms_solver.cu after the Krylov drivers.
#pragma once

namespace cms {

// Compass table of the 5-point solvers: for device row r and k = 0 N, 1 E,
// 2 S, 3 W the device row of the neighbour (-1: dummy).  flags[0]: a cell
// without exactly four faces; flags[1]: a south/west neighbour numbered after
// the cell or a north/east one numbered before it (the order sip.f90 assumes).
__global__ void k_compass(int n, int nmf, const int* __restrict__ perm, const int* __restrict__ iperm,
                          const int* __restrict__ c2c, const int* __restrict__ ncface, int* __restrict__ cmp,
                          int* flags) {
  for (int r = blockIdx.x * TPB + threadIdx.x; r < n; r += gridDim.x * TPB) {
    const int i = perm[r];
    if (ncface[i] != 4) atomicOr(&flags[0], 1);
    for (int k = 0; k < 4; ++k) {
      const int nb = k < nmf ? c2c[(size_t)i * nmf + k] : 0;
      const int j = (nb >= 1 && nb <= n) ? iperm[nb - 1] : -1;
      cmp[(size_t)k * n + r] = j;
      if (j >= 0 && ((k >= 2) != (nb - 1 < i))) atomicOr(&flags[1], 1);
    }
  }
}

enum : int { LEG_FIVE_POINT = 1, LEG_SIP_ORDER = 2 };

// Builds the compass table once per handle; returns the LEG_* properties.
static int legacy_props(Solver* S) {
  if (S->leg_props >= 0) return S->leg_props;
  const HostPattern& P = S->hp;
  CHK(S->alloc(&S->d_cmp, (size_t)4 * P.n));
  int* d_flags = nullptr;
  CHK(S->alloc(&d_flags, 2));
  KLAUNCH(S, P_SCALAR, (double)P.n * 40,
          (k_compass<<<gsz(P.n), TPB, 0, S->stream>>>(P.n, P.nmf, S->d_perm, S->d_iperm, S->d_c2c, S->d_ncface,
                                                       S->d_cmp, d_flags)));
  int h[2] = {0, 0};
  CMS_CUDA(cudaMemcpyAsync(h, d_flags, sizeof(h), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  int props = 0;
  if (!h[0] && P.nmf >= 4) props |= LEG_FIVE_POINT;
  if ((props & LEG_FIVE_POINT) && !h[1] && S->opts.ordering == CMS_ORDER_NATURAL) props |= LEG_SIP_ORDER;
  S->leg_props = props;
  return props;
}

// Per-precision scratch of the 5-point solvers: cf[4n], lw, ls, lpr, un, ue, d.
template <typename T>
static T* legacy_scratch(Solver* S) {
  T*& p = *reinterpret_cast<T**>(sizeof(T) == 8 ? (void*)&S->leg64 : (void*)&S->leg32);
  if (!p && S->alloc(&p, (size_t)10 * S->hp.n) != CMS_OK) return nullptr;
  return p;
}

// Orderings with more groups than this run their recurrences as pipelined
// passes (one launch per pass, or per Gauss-Seidel solve) instead of one
// launch per group.
constexpr int kPipeMinGroups = 16;

static bool use_pipe(const Solver* S) { return S->hp.G > kPipeMinGroups; }

// Chunk table of the pipelined passes (built on first use): every group cut
// into chunks of at most TPB rows.
static int pipe_prepare(Solver* S) {
  const HostPattern& P = S->hp;
  if (!S->d_pipe_cstart) {
    std::vector<int> cs;
    S->pipe_gchunk.assign(P.G + 1, 0);
    for (int g = 0; g < P.G; ++g) {
      S->pipe_gchunk[g] = (int)cs.size();
      for (int r = P.gstart[g]; r < P.gstart[g + 1]; r += TPB) cs.push_back(r);
    }
    S->pipe_gchunk[P.G] = (int)cs.size();
    cs.push_back(P.n);
    S->pipe_nchunk = (int)cs.size() - 1;
    // largest step in groups from a row to an upper neighbour
    std::vector<int> grp(P.n);
    for (int g = 0; g < P.G; ++g)
      for (int r = P.gstart[g]; r < P.gstart[g + 1]; ++r) grp[r] = g;
    int jump = 1;
    for (int r = 0; r < P.n; ++r)
      for (int t = 0; t < P.nup[r]; ++t) jump = std::max(jump, grp[P.col[(size_t)(P.KL + t) * P.n + r]] - grp[r]);
    S->pipe_wave = jump + 1;
    CHK(S->alloc(&S->d_pipe_cstart, cs.size()));
    CMS_CUDA(cudaMemcpyAsync(S->d_pipe_cstart, cs.data(), cs.size() * sizeof(int), cudaMemcpyHostToDevice,
                             S->stream));
    CHK(S->alloc(&S->d_pipe_done, P.n));
    CHK(S->alloc(&S->d_pipe_ticket, 1));
    CHK(S->alloc(&S->d_pipe_err, 8));
    CMS_CUDA(cudaStreamSynchronize(S->stream));
  }
  return CMS_OK;
}

// Start of a solve that uses pipelined passes: pass counts and error flag cleared.
static int pipe_begin(Solver* S) {
  CHK(pipe_prepare(S));
  CMS_CUDA(cudaMemsetAsync(S->d_pipe_done, 0, sizeof(unsigned int) * S->hp.n, S->stream));
  CMS_CUDA(cudaMemsetAsync(S->d_pipe_err, 0, 8 * sizeof(int), S->stream));
  S->pipe_epoch = 0;
  return CMS_OK;
}

// Units of npass forward passes in wavefront order: unit (pass h, chunk of
// group g) in wave g + K h, K = 1 + the largest group step to an upper
// neighbour.  Every unit a unit waits on -- lower neighbours in the same pass,
// upper neighbours and the row itself in the previous one -- is in an earlier
// wave, so the in-order claims cannot wait on an unclaimed unit.
static int pipe_units(Solver* S, int npass) {
  if (S->pipe_units_npass == npass) return CMS_OK;
  const HostPattern& P = S->hp;
  const int K = S->pipe_wave;
  std::vector<int2> u;
  u.reserve((size_t)npass * S->pipe_nchunk);
  const long long waves = (long long)(P.G - 1) + (long long)K * (npass - 1) + 1;
  for (long long d = 0; d < waves; ++d)
    for (int h = 0; h < npass; ++h) {
      const long long g = d - (long long)K * h;
      if (g < 0) break;
      if (g >= P.G) continue;
      for (int c = S->pipe_gchunk[g]; c < S->pipe_gchunk[g + 1]; ++c) u.push_back(make_int2(h, c));
    }
  if (u.size() > S->pipe_units_cap) {
    CHK(S->alloc(&S->d_pipe_units, u.size()));
    S->pipe_units_cap = u.size();
  }
  CMS_CUDA(cudaMemcpyAsync(S->d_pipe_units, u.data(), u.size() * sizeof(int2), cudaMemcpyHostToDevice, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  S->pipe_units_npass = npass;
  return CMS_OK;
}

static PipeSched pipe_sched(Solver* S) {
  return PipeSched{S->d_pipe_cstart, S->pipe_nchunk, S->d_pipe_done, S->d_pipe_ticket, S->d_pipe_err, kSpinLimit};
}


// End of such a solve: a wait that ran out is a device error.
static int pipe_end(Solver* S) {
  int err[8] = {0};
  CMS_CUDA(cudaMemcpyAsync(err, S->d_pipe_err, sizeof(err), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  if (err[0]) {
    std::snprintf(g_last_error, sizeof(g_last_error),
                  "pipelined sweep: row %d timed out waiting for row %d to complete %d passes (saw %d; unit %d of "
                  "%d chunks)", err[1], err[2], err[3], err[4], err[5], S->pipe_nchunk);
    return CMS_DEVICE_ERROR;
  }
  return CMS_OK;
}

// Runs the pipelined passes' wait on a row that never completes, with a
// limit of spin_limit polls: the wait must give up, record where, and leave
// the device usable.  CMS_DEVICE_ERROR (with the message) is the expected
// result; anything else means the bounded wait failed.
static int pipe_wait_selftest(Solver* S, unsigned int spin_limit) {
  CHK(pipe_begin(S));
  PipeSched ps = pipe_sched(S);
  ps.spin_limit = spin_limit;
  KLAUNCH(S, P_SCALAR, 0, (k_pipe_wait_probe<<<1, 32, 0, S->stream>>>(ps, 0)));
  const int rc = pipe_end(S);
  CMS_CUDA(cudaGetLastError());
  return rc;
}

// One pipelined pass of a triangular recurrence (forward: lower slots first).
template <class Op>
static int tri_pipe(Solver* S, const Op& op, bool bwd, double bytes, int cat) {
  const HostPattern& P = S->hp;
  CMS_CUDA(cudaMemsetAsync(S->d_pipe_ticket, 0, sizeof(unsigned int), S->stream));
  const unsigned int epoch = ++S->pipe_epoch;
  const int grid = std::max(1, std::min(S->pipe_nchunk, GRID_CAP));
  KLAUNCH(S, cat, bytes,
          (k_tri_pipe<Op><<<grid, TPB, 0, S->stream>>>(op, P.n, P.KL, S->d_col, S->d_nlo, S->d_nup, pipe_sched(S),
                                                        bwd ? 1 : 0, epoch, S->d_st)));
  return CMS_OK;
}

// One Gauss-Seidel pass over all groups, forward or backward.
template <typename T>
static int gs_pass(Solver* S, Mat<T>& A, Work<T>& W, bool backward, bool sor, T w) {
  const HostPattern& P = S->hp;
  const double s = sizeof(T);
  for (int q = 0; q < P.G; ++q) {
    const int g = backward ? P.G - 1 - q : q;
    const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
    if (r1 <= r0) continue;
    const double R = r1 - r0, E = (double)(P.glo[g] + P.gup[g]);
    if (sor)
      KLAUNCH(S, P_FWD, R * s * 4 + E * (2 * s + 4),
              (k_gs<T, true><<<gsz(r1 - r0), TPB, 0, S->stream>>>(P.n, r0, r1, P.KL, P.gkl[g], P.gku[g], S->d_col,
                                                                    S->d_nlo, S->d_nup, A.aoff, A.diag, W.b, W.x,
                                                                    w)));
    else
      KLAUNCH(S, P_FWD, R * s * 4 + E * (2 * s + 4),
              (k_gs<T, false><<<gsz(r1 - r0), TPB, 0, S->stream>>>(P.n, r0, r1, P.KL, P.gkl[g], P.gku[g], S->d_col,
                                                                     S->d_nlo, S->d_nup, A.aoff, A.diag, W.b, W.x,
                                                                     w)));
  }
  return CMS_OK;
}

// nsweeps forward passes, or nsweeps/2 forward+backward pairs.
template <typename T>
static int run_gauss_seidel(Solver* S, Mat<T>& A, Work<T>& W, int nsweeps, bool symmetric, bool sor, double w,
                            int* done_sweeps) {
  const int reps = symmetric ? nsweeps / 2 : nsweeps;
  if (use_pipe(S) && reps > 0) {  // every pass in one pipelined launch
    const HostPattern& P = S->hp;
    CHK(pipe_begin(S));
    CMS_CUDA(cudaMemsetAsync(S->d_pipe_ticket, 0, sizeof(unsigned int), S->stream));
    const int npass = symmetric ? 2 * reps : reps;
    const int grid = std::max(1, std::min(npass * S->pipe_nchunk, GRID_CAP));
    const int2* units = nullptr;  // alternating passes turn at the ends: pass-major order
    if (!symmetric) {
      CHK(pipe_units(S, npass));
      units = S->d_pipe_units;
    }
    const double bytes = (double)npass * ((double)P.n * sizeof(T) * 4 + (double)P.nnz_off * (2 * sizeof(T) + 4));
    if (sor)
      KLAUNCH(S, P_FWD, bytes,
              (k_gs_pipe<T, true><<<grid, TPB, 0, S->stream>>>(P.n, P.KL, S->d_col, S->d_nlo, S->d_nup, A.aoff,
                                                                A.diag, W.b, W.x, (T)w, pipe_sched(S), npass,
                                                                symmetric ? 1 : 0, 0u, units)));
    else
      KLAUNCH(S, P_FWD, bytes,
              (k_gs_pipe<T, false><<<grid, TPB, 0, S->stream>>>(P.n, P.KL, S->d_col, S->d_nlo, S->d_nup, A.aoff,
                                                                 A.diag, W.b, W.x, (T)w, pipe_sched(S), npass,
                                                                 symmetric ? 1 : 0, 0u, units)));
    CHK(pipe_end(S));
    *done_sweeps = reps;
    return CMS_OK;
  }
  for (int it = 0; it < reps; ++it) {
    CHK(gs_pass<T>(S, A, W, false, sor, (T)w));
    if (symmetric) CHK(gs_pass<T>(S, A, W, true, sor, (T)w));
  }
  *done_sweeps = std::max(reps, 0);
  return CMS_OK;
}

// Diagonal incomplete Cholesky factor into d (group by group).
template <typename T, bool STAB>
static int dic_factor(Solver* S, Mat<T>& A, T* d) {
  const HostPattern& P = S->hp;
  if (use_pipe(S)) {
    OpDicFactor<T, STAB> op{P.n, S->d_col, S->d_nlo, A.aoff, A.diag, d};
    return tri_pipe(S, op, false, (double)P.n * 2 * sizeof(T) + (double)P.nnz_off * (sizeof(T) + 2), P_ILU0);
  }
  for (int g = 0; g < P.G; ++g) {
    const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
    if (r1 <= r0) continue;
    KLAUNCH(S, P_ILU0, (double)(r1 - r0) * 2 * sizeof(T) + (double)P.glo[g] * (2 * sizeof(T) + 4),
            (k_dic<T, STAB><<<gsz(r1 - r0), TPB, 0, S->stream>>>(P.n, r0, r1, P.gkl[g], S->d_col, S->d_nlo, A.aoff,
                                                                  A.diag, d)));
  }
  return CMS_OK;
}

// z = M^-1 y with the diagonal incomplete factor d (iccg.f90:71-79).
template <typename T>
static int dic_apply(Solver* S, Mat<T>& A, const T* d, const T* y, T* z, T eps) {
  const HostPattern& P = S->hp;
  const double s = sizeof(T);
  if (use_pipe(S)) {
    const double half = (double)P.n * s * 3 + (double)P.nnz_off * 0.5 * (s + 4);
    CHK(tri_pipe(S, OpDicFwd<T>{P.n, S->d_col, S->d_nlo, A.aoff, d, y, z}, false, half, P_FWD));
    return tri_pipe(S, OpDicBwd<T>{P.n, P.KL, S->d_col, S->d_nup, A.aoff, d, z, eps}, true, half, P_BWD);
  }
  for (int g = 0; g < P.G; ++g) {
    const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
    if (r1 <= r0) continue;
    KLAUNCH(S, P_FWD, (double)(r1 - r0) * s * 3 + (double)P.glo[g] * (s + 4),
            (k_dic_fwd<T><<<gsz(r1 - r0), TPB, 0, S->stream>>>(P.n, r0, r1, P.gkl[g], S->d_col, S->d_nlo, A.aoff, d,
                                                                y, z, S->d_st)));
  }
  for (int g = P.G - 1; g >= 0; --g) {
    const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
    if (r1 <= r0) continue;
    KLAUNCH(S, P_BWD, (double)(r1 - r0) * s * 3 + (double)P.gup[g] * (s + 4),
            (k_dic_bwd<T><<<gsz(r1 - r0), TPB, 0, S->stream>>>(P.n, r0, r1, P.KL, P.gku[g], S->d_col, S->d_nup,
                                                                A.aoff, d, z, eps, S->d_st)));
  }
  return CMS_OK;
}

// Issues iterations in growing chunks and stops once the device test fired.
template <typename F>
static int legacy_loop(Solver* S, int maxit, F&& iter) {
  int issued = 0, chunk = S->prof_on ? 1 : 2;
  while (issued < maxit) {
    const int c = std::min(chunk, maxit - issued);
    for (int q = 0; q < c; ++q) CHK(iter());
    issued += c;
    bool done = false;
    CHK(poll_done(S, done));
    if (done) break;
    if (!S->prof_on) chunk = std::min(chunk * 2, 16);
  }
  return CMS_OK;
}

// ICCG (iccg.f90:2-184).
template <typename T>
static int run_iccg(Solver* S, Mat<T>& A, Work<T>& W, int maxit) {
  const HostPattern& P = S->hp;
  const int n = P.n, nb_all = S->tab.blk[S->tab.ng];
  T* d = legacy_scratch<T>(S);
  if (!d) return CMS_DEVICE_ERROR;
  d += (size_t)9 * n;
  if (use_pipe(S)) CHK(pipe_begin(S));
  CMS_CUDA(cudaMemsetAsync(W.p, 0, sizeof(T) * n, S->stream));
  CMS_CUDA(cudaMemsetAsync(W.z, 0, sizeof(T) * n, S->stream));
  KLAUNCH(S, P_SCALAR, 0, (k_leg_start<<<1, 1, 0, S->stream>>>(S->d_st, maxit)));
  KLAUNCH(S, P_RESID64, spmv_bytes<T>(S, 3),
          (k_leg_resid<T, LEG_RES_L1><<<nb_all, TPB, 0, S->stream>>>(n, P.KL, S->tab, S->d_col, S->d_nlo, S->d_nup,
                                                                      A.aoff, A.diag, W.b, W.x, W.r, nullptr, 0,
                                                                      S->d_part, S->d_st)));
  CHK((dic_factor<T, false>(S, A, d)));
  const int nitermin = maxit / 2;
  const double vb = (double)n * sizeof(T);
  CHK(legacy_loop(S, maxit, [&]() -> int {
    CHK(dic_apply<T>(S, A, d, W.r, W.z, T(0)));
    KLAUNCH(S, P_VEC, vb * 2, (k_leg_dot<T, LD_ICCG_SK><<<gsz(n), TPB, 0, S->stream>>>(n, W.r, W.z, S->d_part,
                                                                                      S->d_st)));
    KLAUNCH(S, P_VEC, vb * 3, (k_leg_vec<T, LV_ICCG_P><<<gsz(n), TPB, 0, S->stream>>>(n, W.x, W.r, W.p, W.z,
                                                                                     nullptr, S->d_st)));
    KLAUNCH(S, P_SPMV, spmv_bytes<T>(S, 2),
            (k_leg_spmv<T, LS_ICCG><<<nb_all, TPB, 0, S->stream>>>(n, P.KL, S->tab, S->d_col, S->d_nlo, S->d_nup,
                                                                    A.aoff, A.diag, W.p, W.z, W.p, S->d_part,
                                                                    S->d_st)));
    KLAUNCH(S, P_VEC, vb * 6, (k_leg_update<T, true><<<gsz(n), TPB, 0, S->stream>>>(n, W.x, W.r, W.p, W.z, nitermin,
                                                                                   S->d_part, S->d_st)));
    return CMS_OK;
  }));
  return use_pipe(S) ? pipe_end(S) : CMS_OK;
}

// ICCGSTAB (iccgstab.f90:2-163).
template <typename T>
static int run_iccgstab(Solver* S, Mat<T>& A, Work<T>& W, int maxit) {
  const HostPattern& P = S->hp;
  const int n = P.n, nb_all = S->tab.blk[S->tab.ng];
  T* d = legacy_scratch<T>(S);
  if (!d) return CMS_DEVICE_ERROR;
  d += (size_t)9 * n;
  if (use_pipe(S)) CHK(pipe_begin(S));
  T* zero[4] = {W.p, W.u, W.z, W.v};
  for (int q = 0; q < 4; ++q) {
    CMS_CUDA(cudaMemsetAsync(zero[q], 0, sizeof(T) * n, S->stream));
  }
  KLAUNCH(S, P_SCALAR, 0, (k_leg_start<<<1, 1, 0, S->stream>>>(S->d_st, maxit)));
  KLAUNCH(S, P_SCALAR, 0, (k_stab_start<<<1, 1, 0, S->stream>>>(S->d_st)));
  KLAUNCH(S, P_RESID64, spmv_bytes<T>(S, 4),
          (k_leg_resid<T, LEG_RES_L1_COPY><<<nb_all, TPB, 0, S->stream>>>(n, P.KL, S->tab, S->d_col, S->d_nlo,
                                                                           S->d_nup, A.aoff, A.diag, W.b, W.x, W.r,
                                                                           W.r0, 0, S->d_part, S->d_st)));
  CHK((dic_factor<T, true>(S, A, d)));
  const T eps = T(1.0e-20);
  const double vb = (double)n * sizeof(T);
  CHK(legacy_loop(S, maxit, [&]() -> int {
    KLAUNCH(S, P_VEC, vb * 2, (k_leg_dot<T, LD_STAB_BET><<<gsz(n), TPB, 0, S->stream>>>(n, W.r, W.r0, S->d_part,
                                                                                       S->d_st)));
    KLAUNCH(S, P_VEC, vb * 4, (k_leg_vec<T, LV_STAB_P><<<gsz(n), TPB, 0, S->stream>>>(n, W.x, W.r, W.p, nullptr,
                                                                                     W.u, S->d_st)));
    CHK(dic_apply<T>(S, A, d, W.p, W.z, eps));
    KLAUNCH(S, P_SPMV, spmv_bytes<T>(S, 3),
            (k_leg_spmv<T, LS_STAB_U><<<nb_all, TPB, 0, S->stream>>>(n, P.KL, S->tab, S->d_col, S->d_nlo, S->d_nup,
                                                                      A.aoff, A.diag, W.z, W.u, W.r0, S->d_part,
                                                                      S->d_st)));
    KLAUNCH(S, P_VEC, vb * 6, (k_leg_vec<T, LV_STAB_X><<<gsz(n), TPB, 0, S->stream>>>(n, W.x, W.r, nullptr, W.z,
                                                                                     W.u, S->d_st)));
    CHK(dic_apply<T>(S, A, d, W.r, W.z, eps));
    KLAUNCH(S, P_SPMV, spmv_bytes<T>(S, 3),
            (k_leg_spmv<T, LS_STAB_V><<<nb_all, TPB, 0, S->stream>>>(n, P.KL, S->tab, S->d_col, S->d_nlo, S->d_nup,
                                                                      A.aoff, A.diag, W.z, W.v, W.r, S->d_part,
                                                                      S->d_st)));
    KLAUNCH(S, P_VEC, vb * 6, (k_leg_update<T, false><<<gsz(n), TPB, 0, S->stream>>>(n, W.x, W.r, W.z, W.v, 0,
                                                                                    S->d_part, S->d_st)));
    return CMS_OK;
  }));
  return use_pipe(S) ? pipe_end(S) : CMS_OK;
}

// SIP (sip.f90:2-174).  acoef: the caller's natural-order array, or with
// face_nD > 0 the flow's face coefficients ([nmf][face_nD], device rows).
template <typename T>
static int run_sip(Solver* S, Mat<T>& A, Work<T>& W, const T* acoef, int maxit, int face_nD = 0) {
  const HostPattern& P = S->hp;
  const int n = P.n, nb_all = S->tab.blk[S->tab.ng];
  T* base = legacy_scratch<T>(S);
  if (!base) return CMS_DEVICE_ERROR;
  T* cf = base;
  SipFactor<T> f{base + (size_t)4 * n, base + (size_t)5 * n, base + (size_t)6 * n, base + (size_t)7 * n,
                 base + (size_t)8 * n};
  const double s = sizeof(T);
  if (face_nD > 0)
    KLAUNCH(S, P_VEC, (double)n * 8 * s,
            (k_sip_coef_dev<T><<<gsz(n), TPB, 0, S->stream>>>(n, face_nD, acoef, cf)));
  else
    KLAUNCH(S, P_VEC, (double)n * (4 + 8 * s),
            (k_sip_coef<T><<<gsz(n), TPB, 0, S->stream>>>(n, P.nmf, S->d_perm, acoef, cf)));
  const bool pipe = use_pipe(S);
  // counters first: the pipelined factor pass below skips itself while the
  // previous solve's stop flag is still set
  KLAUNCH(S, P_SCALAR, 0, (k_leg_start<<<1, 1, 0, S->stream>>>(S->d_st, maxit)));
  if (pipe) {
    CHK(pipe_begin(S));
    CHK(tri_pipe(S, OpSipFactor<T>{n, S->d_cmp, cf, A.diag, f, T(0.92)}, false, (double)n * (16 + 14 * s), P_ILU0));
  } else {
    for (int g = 0; g < P.G; ++g) {
      const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
      if (r1 <= r0) continue;
      KLAUNCH(S, P_ILU0, (double)(r1 - r0) * (16 + 14 * s),
              (k_sip_factor<T><<<gsz(r1 - r0), TPB, 0, S->stream>>>(n, r0, r1, S->d_cmp, cf, A.diag, f, T(0.92))));
    }
  }
  const int nitermin = maxit / 2;
  CHK(legacy_loop(S, maxit, [&]() -> int {
    KLAUNCH(S, P_RESID64, spmv_bytes<T>(S, 3),
            (k_leg_resid<T, LEG_SIP_RES><<<nb_all, TPB, 0, S->stream>>>(n, P.KL, S->tab, S->d_col, S->d_nlo,
                                                                         S->d_nup, A.aoff, A.diag, W.b, W.x, W.r,
                                                                         nullptr, nitermin, S->d_part, S->d_st)));
    if (pipe) {
      CHK(tri_pipe(S, OpSipFwd<T>{n, S->d_cmp, f, W.r, W.z}, false, (double)n * (8 + 6 * s), P_FWD));
      CHK(tri_pipe(S, OpSipBwd<T>{n, S->d_cmp, f, W.z}, true, (double)n * (8 + 6 * s), P_BWD));
    } else {
      for (int g = 0; g < P.G; ++g) {
        const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
        if (r1 <= r0) continue;
        KLAUNCH(S, P_FWD, (double)(r1 - r0) * (8 + 6 * s),
                (k_sip_fwd<T><<<gsz(r1 - r0), TPB, 0, S->stream>>>(n, r0, r1, S->d_cmp, f, W.r, W.z, S->d_st)));
      }
      for (int g = P.G - 1; g >= 0; --g) {
        const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
        if (r1 <= r0) continue;
        KLAUNCH(S, P_BWD, (double)(r1 - r0) * (8 + 6 * s),
                (k_sip_bwd<T><<<gsz(r1 - r0), TPB, 0, S->stream>>>(n, r0, r1, S->d_cmp, f, W.z, S->d_st)));
      }
    }
    KLAUNCH(S, P_VEC, (double)n * s * 3,
            (k_leg_vec<T, LV_SIP_ADD><<<gsz(n), TPB, 0, S->stream>>>(n, W.x, nullptr, nullptr, W.z, nullptr,
                                                                     S->d_st)));
    KLAUNCH(S, P_SCALAR, 0, (k_leg_finish<<<1, 1, 0, S->stream>>>(S->d_st)));
    return CMS_OK;
  }));
  return pipe ? pipe_end(S) : CMS_OK;
}

// Which method a legacy nsolv runs for variable n (solvers.f90:242-289).
enum LegKind : int { LK_KRYLOV = 0, LK_GS = 1, LK_SIP = 2, LK_ICCG = 3, LK_ICCGSTAB = 4, LK_NONE = 5 };

struct LegPlan {
  int kind = LK_KRYLOV;
  int sweeps = 0;        // Gauss-Seidel passes (symmetric: pairs x 2)
  bool symmetric = false;
  bool sor = false;
};

// rmom: the RMS normalised residual of this call (rmom(n); the pressure
// branches read rmom(1) only when n == 1).
static LegPlan legacy_plan(int nsolv, int n, double rmom, int nswp, int nswp0_vel) {
  LegPlan p;
  switch (nsolv) {
    case 0: p.kind = LK_NONE; break;  // ADI: solve() has no branch for it
    case 1: p.kind = LK_GS; p.sweeps = nswp; break;
    case 2:
      p.kind = LK_GS; p.sweeps = nswp; p.symmetric = true; p.sor = n == 1 && rmom < 1.0e-3;
      break;
    case 5:
      if (n == 1 && rmom > 1.0e-4) break;  // pbicgstab with nswp(1)
      p.kind = LK_GS;
      p.sweeps = n >= 4 ? 3 * nswp0_vel : 4 * nswp;  // nswp(1:3) = 4 nswp0, nswp(4:5) = 3 nswp0(2:3)
      p.sor = n == 1 && rmom < 1.0e-3;
      break;
    case 6: p.kind = LK_SIP; break;
    case 7: p.kind = n == 1 ? LK_ICCG : LK_SIP; break;
    case 8: p.kind = n == 1 ? LK_ICCG : LK_ICCGSTAB; break;
    default: break;
  }
  return p;
}

}  // namespace cms
