// Ensemble of independent flow models stepped together (included at the end
// of cms_solver.cu after the flow host code).
//
// The members advance their outer SIMPLEC iterations in lockstep: each stage
// of the step runs for every member still iterating, each member on its own
// stream, and each of the three Krylov solves of an outer iteration is one
// batched persistent launch for all members (k_bicg_batched): every member
// keeps its own tiles, tile waits, barrier, dot products and stopping test,
// so a member's result does not depend on the others.  A member leaves the
// loop when its check_conv says so, exactly as in its own step.
//
// Layout: the launch's blocks (at most the device's resident capacity) are
// split among the members in proportion to their unknowns, at least one
// each; cms_ensemble_set_tiles picks the total (the autotuner in
// cms2d_b200/ensemble.py times the candidates).
#pragma once

struct cms_ensemble {
  std::vector<cms_flow*> m;
  int dev = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_done = nullptr;
  std::vector<cudaEvent_t> ev_m;
  std::vector<int> tiles;  // per member
  int total_tiles = 0;
  int batched = 0;  // 1: the solves run as batched persistent launches
  cms::PersistArgs<float>* d_args = nullptr;
  cms::PersistArgs<float>* h_args = nullptr;  // pinned
  cms::SchurArgs* d_sargs = nullptr;           // reduced inner solves (every member in reduced form)
  cms::SchurArgs* h_sargs = nullptr;           // pinned
  int2* d_bmap = nullptr;
  int2* h_bmap = nullptr;  // pinned
  long long launches = 0;
};

namespace cms {

using Ens = ::cms_ensemble;

// Splits total blocks among the members by unknowns and builds their tables.
static int ensemble_layout(Ens* E, int total) {
  const int M = (int)E->m.size();
  const int cap = persist_capacity(E->dev);
  if (cap <= 0) return CMS_UNSUPPORTED;
  if (total <= 0 || total > cap) total = cap;
  total = std::max(total, M);
  double nsum = 0.0;
  for (auto* F : E->m) nsum += F->n;
  std::vector<int> t(M);
  int used = 0;
  for (int i = 0; i < M; ++i) {
    t[i] = std::max(1, (int)std::floor(total * (double)E->m[i]->n / nsum));
    t[i] = std::min(t[i], nblk(E->m[i]->n));
    used += t[i];
  }
  while (used > total) {  // trim the largest shares
    int j = (int)(std::max_element(t.begin(), t.end()) - t.begin());
    if (t[j] <= 1) break;
    --t[j];
    --used;
  }
  used = 0;
  for (int i = 0; i < M; ++i) {
    const int got = build_tiles(E->m[i]->S, t[i]);
    if (got <= 0) return CMS_UNSUPPORTED;
    t[i] = got;
    used += got;
  }
  if (used > cap) return CMS_UNSUPPORTED;
  E->tiles = t;
  E->total_tiles = used;
  return CMS_OK;
}

// run_refine for several members at once: FP64 residuals per member, then
// one batched launch for the FP32 inner BiCGStab solves of every member
// that continues.  act: member indices; nswp: iteration caps.  A member whose
// last inner correction made its FP64 residual larger (or overflowed) has it
// undone and finishes on its own with the exact factor (refine_exact).
static int refine_batched(Ens* E, const std::vector<int>& act, const std::vector<int>& nswp,
                          std::vector<cms_solve_info*>& infos) {
  const int A_ = (int)act.size();
  std::vector<RefineState> R(A_);
  std::vector<char> live(A_, 1);
  struct Reset {  // cur_relax describes A32's factor only during this solve
    Ens* e;
    const std::vector<int>& a;
    ~Reset() {
      for (int i : a) {
        e->m[i]->S->cur_relax = 0;
        e->m[i]->S->cur_fuse = 0;
      }
    }
  } reset{E, act};
  // the reduced inner form when every member's solver takes it (as each
  // member's own step does), else the two-phase or exact factor
  bool schur = true;
  for (int j = 0; j < A_ && schur; ++j) {
    Solver* S = E->m[act[j]]->S;
    schur = S->opts.inner_relax == 2 && S->opts.ordering == CMS_ORDER_MULTICOLOR &&
            schur_pattern(S, E->tiles[act[j]]) == CMS_OK;
  }
  // the single-reduction form when every member's layout option asks for it
  // and every member's pattern is symmetric (the launch is one kernel)
  bool sr = schur;
  for (int j = 0; j < A_ && sr; ++j) {
    Solver* S = E->m[act[j]]->S;
    sr = schur_layout(schur_layout_index(S)).sr && S->sc_sym;
  }
  bool relax_any = false;
  for (int j = 0; j < A_; ++j) {
    Solver* S = E->m[act[j]]->S;
    const HostPattern& P = S->hp;
    const int n = P.n;
    RefineState& rm = R[j];
    rm.info = infos[j];
    rm.maxit = S->opts.max_iters > 0 ? S->opts.max_iters : nswp[j];
    rm.tol = S->opts.tol > 0 ? S->opts.tol : 1e-3;
    rm.rmax = S->opts.max_refine > 0 ? S->opts.max_refine : 30;
    const bool relax = S->opts.inner_relax && S->opts.ordering == CMS_ORDER_MULTICOLOR && P.G > 2;
    S->cur_fuse = 1;
    if (schur) {
      CHK(schur_numeric(S));
    } else if (relax) {
      KLAUNCH(S, P_ILU0, (double)n * (3 * 4 + 2) + (double)(P.nnz_off) * (2 * 4 + 4),
              (k_ilu0_relax<float><<<gsz(n), TPB, 0, S->stream>>>(n, P.KL, P.gstart[1], S->d_col, S->d_nlo,
                                                                   S->d_nup, S->A32.aoff, S->A32.diag, S->A32.luoff,
                                                                   S->A32.invd)));
      S->cur_relax = 1;
      relax_any = true;
    } else {
      CHK(factor<float>(S, S->A32));
    }
  }
  const bool inexact = schur || relax_any;
  for (;;) {
    std::vector<int> cont;
    for (int j = 0; j < A_; ++j) {
      if (!live[j]) continue;
      Solver* S = E->m[act[j]]->S;
      bool go = true, worse = false;
      CHK(refine_check(S, R[j], go, worse));
      if (worse) {
        if (go && inexact) CHK(refine_exact(S, 3, R[j]));
        live[j] = 0;
      } else if (!go) {
        live[j] = 0;
      } else {
        cont.push_back(j);
      }
    }
    if (cont.empty()) break;
    // inner FP32 solves A32 d = r/||r|| from d = 0, all members in one launch
    int blocks = 0;
    for (int c = 0; c < (int)cont.size(); ++c) {
      const int j = cont[c], i = act[j];
      Solver* S = E->m[i]->S;
      const int n = S->hp.n;
      KLAUNCH(S, P_VEC, (double)n * 12,
              (k_ir_scale<<<gsz(n), TPB, 0, S->stream>>>(n, S->W64.r, S->W32.b, S->d_st)));
      CMS_CUDA(cudaMemsetAsync(&S->d_st->bar, 0, sizeof(GridBar), S->stream));
      CMS_CUDA(cudaMemsetAsync(S->d_progress, 0, sizeof(unsigned int) * E->tiles[i] * kProgressStride, S->stream));
      refine_inner_limits(S->opts, R[j]);
      if (schur) E->h_sargs[c] = make_schur_args(S, E->tiles[i], R[j].imax, R[j].itol);
      else E->h_args[c] = make_args<float>(S, S->A32, S->W32, E->tiles[i], R[j].imax, 2, R[j].itol, 1);
      for (int t = 0; t < E->tiles[i]; ++t) E->h_bmap[blocks++] = make_int2(c, t);
      CMS_CUDA(cudaEventRecord(E->ev_m[i], S->stream));
      CMS_CUDA(cudaStreamWaitEvent(E->stream, E->ev_m[i], 0));
    }
    if (schur)
      CMS_CUDA(cudaMemcpyAsync(E->d_sargs, E->h_sargs, cont.size() * sizeof(SchurArgs), cudaMemcpyHostToDevice,
                               E->stream));
    else
      CMS_CUDA(cudaMemcpyAsync(E->d_args, E->h_args, cont.size() * sizeof(PersistArgs<float>),
                               cudaMemcpyHostToDevice, E->stream));
    CMS_CUDA(cudaMemcpyAsync(E->d_bmap, E->h_bmap, blocks * sizeof(int2), cudaMemcpyHostToDevice, E->stream));
    if (schur) {
      void* kargs[] = {&E->d_sargs, &E->d_bmap};
      // the layout the ensemble's tile split was sized for (256 threads per block)
      const void* kern = sr ? (const void*)k_schur_batched<TPB, 2, 1> : (const void*)k_schur_batched<TPB, 2, 0>;
      CMS_CUDA(cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(TPB), kargs, 0, E->stream));
    } else {
      void* kargs[] = {&E->d_args, &E->d_bmap};
      CMS_CUDA(cudaLaunchCooperativeKernel((const void*)k_bicg_batched<float>, dim3(blocks), dim3(TPB), kargs, 0,
                                           E->stream));
    }
    E->launches++;
    CMS_CUDA(cudaEventRecord(E->ev_done, E->stream));
    for (int j : cont) {
      Solver* S = E->m[act[j]]->S;
      CMS_CUDA(cudaStreamWaitEvent(S->stream, E->ev_done, 0));
      CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
    }
    for (int j : cont) {
      Solver* S = E->m[act[j]]->S;
      CMS_CUDA(cudaStreamSynchronize(S->stream));
      if (S->h_st->bar.err) {
        std::snprintf(g_last_error, sizeof(g_last_error), "batched BiCGStab: a wait timed out");
        return CMS_DEVICE_ERROR;
      }
      R[j].inner_total += S->h_st->iter;
      if (S->h_st->nonfinite) {  // no correction from an overflowed inner solve (as run_refine)
        if (inexact) CHK(refine_exact(S, 3, R[j]));
        live[j] = 0;
        continue;
      }
      CHK(refine_correct(S, R[j]));
    }
  }
  for (int j = 0; j < A_; ++j) {
    Solver* S = E->m[act[j]]->S;
    CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
  }
  for (int j = 0; j < A_; ++j) {
    Solver* S = E->m[act[j]]->S;
    CMS_CUDA(cudaStreamSynchronize(S->stream));
    refine_finish(R[j]);
    R[j].info->rmom = S->h_st->s[S_RMOM];
  }
  return CMS_OK;
}

enum EnsSystem { ES_U = 0, ES_V = 1, ES_PP = 2 };

// One of the three solves of an outer iteration for the members in act.
static int ensemble_solve(Ens* E, const std::vector<int>& act, int which) {
  std::vector<cms_solve_info*> infos(act.size());
  std::vector<int> nswp(act.size());
  for (size_t j = 0; j < act.size(); ++j) {
    Flow* F = E->m[act[j]];
    FlowState& T = F->st;
    cms_solve_info* si = &F->last_solve[which];
    std::memset(si, 0, sizeof(*si));
    si->ncolors = F->S->hp.G;
    si->true_relres = -1.0;
    infos[j] = si;
    if (which == ES_U) CHK(flow_solve_begin(F, T.su, T.spu, T.u, F->G.relax_uv));
    else if (which == ES_V) CHK(flow_solve_begin(F, T.sv, T.spv, T.v, F->G.relax_uv));
    else CHK(flow_solve_begin(F, T.su, T.sp, T.pp, 1.0));
    nswp[j] = which == ES_PP ? F->opts.nswp_pp : F->opts.nswp_uv;
  }
  if (E->batched) {
    CHK(refine_batched(E, act, nswp, infos));
  } else {
    for (size_t j = 0; j < act.size(); ++j) {
      Flow* F = E->m[act[j]];
      const int nvar = which == ES_U ? 2 : which == ES_V ? 3 : 1;
      const int rc = solve_core64(F->S, F->opts.nsolv, nswp[j], infos[j], nvar, F->st.acoef, F->nD);
      if (rc == CMS_DEVICE_ERROR || rc == CMS_UNSUPPORTED || rc == CMS_BAD_ARGUMENT) return rc;
    }
  }
  for (size_t j = 0; j < act.size(); ++j) {
    Flow* F = E->m[act[j]];
    FlowState& T = F->st;
    double* phi = which == ES_U ? T.u : which == ES_V ? T.v : T.pp;
    double* rm = which == ES_U ? &F->it_rm[2] : which == ES_V ? &F->it_rm[3] : &F->it_rm[1];
    CHK(flow_solve_end(F, phi, rm, infos[j]));
    F->it_kry += infos[j]->iters;
  }
  return CMS_OK;
}

static int ensemble_step(Ens* E, double dt, const double* const* wsebnd, cms_flow_info* infos) {
  const int M = (int)E->m.size();
  std::vector<int> niter(M, 0), iconv(M, 1), done(M, 0), maxit(M);
  for (int i = 0; i < M; ++i) {
    CHK(step_begin(E->m[i], dt, wsebnd ? wsebnd[i] : nullptr));
    maxit[i] = flow_maxit(E->m[i]);
  }
  for (int it = 1;; ++it) {
    std::vector<int> act;
    for (int i = 0; i < M; ++i)
      if (!done[i] && it <= maxit[i]) act.push_back(i);
    if (act.empty()) break;
    for (int i : act) {
      niter[i] = it;
      CHK(stage_uv(E->m[i]));
    }
    CHK(ensemble_solve(E, act, ES_U));
    auto drop_nonfinite = [&](int which) {
      std::vector<int> keep;
      for (int i : act) {
        if (E->m[i]->last_solve[which].status == CMS_NONFINITE) { iconv[i] = 0; done[i] = 1; }
        else keep.push_back(i);
      }
      act.swap(keep);
    };
    drop_nonfinite(ES_U);
    if (!act.empty()) CHK(ensemble_solve(E, act, ES_V));
    drop_nonfinite(ES_V);
    for (int i : act) CHK(stage_pp(E->m[i]));
    if (!act.empty()) CHK(ensemble_solve(E, act, ES_PP));
    drop_nonfinite(ES_PP);
    for (int i : act) {
      CHK(stage_corr(E->m[i], it, maxit[i], &iconv[i]));
      if (iconv[i] == 0 || iconv[i] == 2) done[i] = 1;
    }
  }
  int status = CMS_OK;
  for (int i = 0; i < M; ++i) {
    cms_flow_info loc{};
    const int rc = step_end(E->m[i], dt, std::min(niter[i], maxit[i]), iconv[i], infos ? &infos[i] : &loc);
    if (rc == CMS_DEVICE_ERROR) return rc;
    if (rc != CMS_OK && status == CMS_OK) status = rc;
  }
  return status;
}

}  // namespace cms

extern "C" {

int cms_ensemble_create(int nmembers, cms_flow* const* members, cms_ensemble** out) {
  if (!out || nmembers <= 0 || !members) return CMS_BAD_ARGUMENT;
  for (int i = 0; i < nmembers; ++i)
    if (!members[i]) return CMS_BAD_ARGUMENT;
  auto* E = new cms_ensemble();
  E->m.assign(members, members + nmembers);
  for (auto* F : E->m) F->use_graphs = 1;  // stage kernel sequences replayed as CUDA graphs
  auto fail = [&](int rc) { cms_ensemble_destroy(E); return rc; };
  if (cudaGetDevice(&E->dev) != cudaSuccess || cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) ||
      cudaEventCreateWithFlags(&E->ev_done, cudaEventDisableTiming))
    return fail(CMS_DEVICE_ERROR);
  E->ev_m.resize(nmembers, nullptr);
  for (auto& e : E->ev_m)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming)) return fail(CMS_DEVICE_ERROR);
  // batched solves: every member FP32 + refinement with persistent BiCGStab
  bool ok = true;
  for (auto* F : E->m) {
    const cms_solver_opts& o = F->S->opts;
    ok = ok && F->opts.nsolv == 3 && o.precision == CMS_PREC_FP32_REFINE && !o.multi_kernel;
  }
  if (ok && nmembers <= cms::GRID_CAP && cms::ensemble_layout(E, 0) == CMS_OK) {
    if (cudaMalloc((void**)&E->d_args, nmembers * sizeof(cms::PersistArgs<float>)) ||
        cudaMallocHost((void**)&E->h_args, nmembers * sizeof(cms::PersistArgs<float>)) ||
        cudaMalloc((void**)&E->d_sargs, nmembers * sizeof(cms::SchurArgs)) ||
        cudaMallocHost((void**)&E->h_sargs, nmembers * sizeof(cms::SchurArgs)) ||
        cudaMalloc((void**)&E->d_bmap, cms::GRID_CAP * sizeof(int2)) ||
        cudaMallocHost((void**)&E->h_bmap, cms::GRID_CAP * sizeof(int2)))
      return fail(CMS_DEVICE_ERROR);
    E->batched = 1;
  }
  *out = E;
  return CMS_OK;
}

int cms_ensemble_set_tiles(cms_ensemble* e, int total_tiles) {
  if (!e) return CMS_BAD_ARGUMENT;
  if (!e->batched) return CMS_UNSUPPORTED;
  return cms::ensemble_layout(e, total_tiles);
}

int cms_ensemble_tiles(const cms_ensemble* e, int* per_member) {
  if (!e) return -1;
  if (per_member)
    for (size_t i = 0; i < e->tiles.size(); ++i) per_member[i] = e->tiles[i];
  return e->total_tiles;
}

int cms_ensemble_batched(const cms_ensemble* e) { return e ? e->batched : 0; }

int cms_ensemble_capacity(const cms_ensemble* e) { return e ? cms::persist_capacity(e->dev) : 0; }

long long cms_ensemble_launches(const cms_ensemble* e) { return e ? e->launches : 0; }

int cms_ensemble_step(cms_ensemble* e, double dt, const double* const* wsebnd, cms_flow_info* infos) {
  if (!e || dt <= 0.0) return CMS_BAD_ARGUMENT;
  for (size_t i = 0; i < e->m.size(); ++i)
    if (!e->m[i]->inited || (e->m[i]->nth > 0 && (!wsebnd || !wsebnd[i]))) return CMS_BAD_ARGUMENT;
  return cms::ensemble_step(e, dt, wsebnd, infos);
}

void cms_ensemble_destroy(cms_ensemble* e) {
  if (!e) return;
  if (e->d_args) cudaFree(e->d_args);
  if (e->h_args) cudaFreeHost(e->h_args);
  if (e->d_sargs) cudaFree(e->d_sargs);
  if (e->h_sargs) cudaFreeHost(e->h_sargs);
  if (e->d_bmap) cudaFree(e->d_bmap);
  if (e->h_bmap) cudaFreeHost(e->h_bmap);
  for (auto ev : e->ev_m)
    if (ev) cudaEventDestroy(ev);
  if (e->ev_done) cudaEventDestroy(e->ev_done);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

}  // extern "C"
