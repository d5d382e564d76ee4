// Host driver of the device flow step (included at the end of cms_solver.cu so
// that it shares the solver's handle internals).
//
// One cms_flow handle owns the grid metrics in device order, the flow state,
// and a solver handle whose device order it adopts, so that the assembly
// kernels write the three systems straight into the solver's matrix buffers.
#pragma once
#include <algorithm>
#include <chrono>
#include <vector>

#include "cms_flow.cuh"
#include "cms_flow_geom.h"
#include "cms_flow_wetdry.h"

struct cms_flow {
  cms_solver* S = nullptr;
  cms::FlowGeom geom;
  cms::FlowDev G{};
  cms::FlowState st{};
  cms_flow_opts opts{};
  int n = 0, nD = 0, nmf = 0;
  std::vector<int> d2n, n2d;  // device <-> natural numbering of all nD cells
  std::vector<void*> allocs;
  size_t bytes = 0;
  // water-level string (device numbering)
  int nth = 0;
  int *d_th_cell = nullptr, *d_th_dummy = nullptr;
  std::vector<int> th_cell_nat, th_dummy_nat;  // the same, natural numbering (0-based)
  double* d_wse = nullptr;       // [nth] values of the current step
  double* d_wse_cell = nullptr;  // [nD] the same, at the dummy cells
  // tidal/harmonic constituents of the string, evaluated on the device when
  // a step is given no water levels (cms_flow_set_tide)
  int ntc = 0;
  double *d_tide = nullptr, *d_psi = nullptr, *d_wsevar = nullptr;  // [ntc][5], [nth][ntc], [nth]
  double tide_dtj = 0.0, tide_offset = 0.0;
  // wall string
  int nw = 0;
  int *d_w_cell = nullptr, *d_w_dummy = nullptr;
  // eddy-viscosity recurrences, level by level (buffers hold up to n cells)
  std::vector<int> wall_lvl, corner_lvl;  // level starts (size levels+1)
  int *d_wall_cells = nullptr, *d_corner_cells = nullptr;
  unsigned char *d_wall_rd = nullptr, *d_corner_rd = nullptr;
  int* d_wall_src = nullptr;    // [n * nmf] per list entry and face slot: wallv face of the dry cell's last writer
  double* d_wallv = nullptr;    // [nmf][nD] value each wall face wrote
  int *d_wall_fin_cells = nullptr, *d_wall_fin_faces = nullptr;  // dry cells written, their last writer's face
  int nwall_fin = 0;
  // wetting and drying: rules, device depth classes, the wet flags (device
  // order) and the wet-cell gradient operator they feed
  cms::WetDryRules wd;
  unsigned char* d_code = nullptr;  // [nD] depth classes of the last evaluation (device order)
  int* d_iwet = nullptr;            // [nD] = G.iwet
  cms::GWOut gw{};
  int wd_pending = 0;               // depth classes changed at the end of the last step
  int inited = 0;                   // cms_flow_init has run (it builds the wet set and its operator)
  int nwet = 0, last_changed = 0;
  long long wd_updates = 0;
  double wd_ms[3] = {0, 0, 0};      // host time of the updates: read-back, rules, application
  int* d_list = nullptr;            // [n + nD] cell lists of an update (device numbering)
  double* d_buf = nullptr;          // [3 nD] gathered (u, v, vis)
  // host copies (natural order) the incremental update works from
  std::vector<unsigned char> code_nat, w0, pn;  // depth classes, depth set, narrow-channel set
  cms::NarrowScratch nsc;
  std::vector<unsigned char> wall_mem;          // [n] wet cells with a face to a dry cell or a dummy
  std::vector<int> wall_list, corner_list;      // eddy-viscosity recurrence cells, cell order
  std::vector<int> vpos, vlast;                 // [n] schedule-builder scratch, -1 between uses
  // device side of the update: narrow-channel set, flow_pond's union-find
  unsigned char* d_pn = nullptr;                // [nD] (device order)
  int* d_par = nullptr;                         // [n] union-find parents
  unsigned char* d_seeded = nullptr;            // [n] component holds a wet string cell
  int* d_seedc = nullptr;                       // string cells (device rows)
  int nseedc = 0;
  int* d_fchg = nullptr;                        // [n] active cells whose final flag changed
  int* d_cnt = nullptr;                         // [1] their count
  int* d_chg = nullptr;                         // [nD] cells whose depth classes changed (kf_wet_codes)
  int nchg_pending = 0;
  signed char* d_fslot_dev = nullptr;  // [nmf][n] ELL slot of face k of device row r
  // gradient copies: index of the current one
  int cur_dppx = 0, cur_duv = 0, cur_dH = 0, cur_dap = 0;
  // CUDA graphs of the stage kernel sequences (pressure-correction assembly,
  // corrections), one per stage and gradient-copy state: a stage's kernels
  // and arguments are fixed for a given state until the wet set changes
  // (graph_gen counts those changes).  use_graphs: replay them (ensembles).
  struct StageGraph {
    cudaGraphExec_t exec = nullptr;
    long long gen = -1;
    int key_after = 0;
    long long nlaunch = 0;
  };
  StageGraph sgraph[2][16];
  int use_graphs = 0;
  long long graph_gen = 0, graph_launches = 0, graph_captures = 0;
  int* h_flag = nullptr;
  cms_flow_info last{};
  cms_solve_info last_solve[3]{};  // u, v, pp of the last outer iteration
  long long launches = 0;
  double t_sim = 0.0;
  double nfaces = 0.0;  // faces of active cells (sum of ncface), for byte counts
  // outer-loop state of the step in progress (check_conv's residual history)
  double it_rm[4] = {0, 0, 0, 0}, it_rmom0[4] = {0, 0, 0, 0}, it_rmom1[4] = {0, 0, 0, 0};
  long long it_kry = 0;

  template <typename P>
  int alloc(P** p, size_t count) {
    const size_t nb = std::max<size_t>(count, 1) * sizeof(P);
    if (cudaMalloc((void**)p, nb) != cudaSuccess) return CMS_DEVICE_ERROR;
    if (cudaMemsetAsync(*p, 0, nb, S->stream) != cudaSuccess) return CMS_DEVICE_ERROR;
    allocs.push_back((void*)*p);
    bytes += nb;
    return CMS_OK;
  }
  template <typename P>
  int upload(P** p, const std::vector<P>& h) {
    int rc = alloc(p, h.size());
    if (rc) return rc;
    if (!h.empty() && cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(P), cudaMemcpyHostToDevice, S->stream))
      return CMS_DEVICE_ERROR;
    return CMS_OK;
  }
};

namespace cms {

using Flow = ::cms_flow;

#define FCHK(...)                     \
  do {                                \
    int rc_ = (__VA_ARGS__);          \
    if (rc_ != CMS_OK) return rc_;    \
  } while (0)

// Launch of a flow kernel with error check, launch count and optional timing
// (profiled under the solver handle's flow class).
#define FLAUNCH(F, ...) FLAUNCHB(F, 0.0, __VA_ARGS__)
#define FLAUNCHB(F, BYTES, ...)                                                                   \
  do {                                                                                            \
    prof_begin((F)->S);                                                                           \
    __VA_ARGS__;                                                                                  \
    (F)->launches++;                                                                              \
    cudaError_t e_ = cudaGetLastError();                                                          \
    if (e_ != cudaSuccess) {                                                                      \
      std::snprintf(g_last_error, sizeof(g_last_error), "flow launch: %s", cudaGetErrorString(e_)); \
      return CMS_DEVICE_ERROR;                                                                    \
    }                                                                                             \
    prof_end((F)->S, P_FLOW, (double)(BYTES));                                                    \
  } while (0)

// Krylov solve of the system a flow prologue wrote into the FP64 buffers
// (A64, W64.b, W64.x; A32 too for refinement); the solution stays in W64.x.
// The solve of a system the flow kernels assembled into the solver's device
// buffers.  nvar: the variable index of solve(..., n) (1 pp, 2 u, 3 v), read
// by the MATRIX_SOLVER options other than BiCGStab and GMRES; face: the flow's
// face coefficients ([nmf][nD], device rows), from which SIP takes its compass
// coefficients.
static int solve_core64(Solver* S, int nsolv, int nswp, cms_solve_info* info, int nvar = 0,
                        const double* face = nullptr, int nD = 0) {
  std::memset(info, 0, sizeof(*info));
  info->ncolors = S->hp.G;
  info->true_relres = -1.0;
  if (nsolv < 0 || nsolv > 8) return info->status = CMS_UNSUPPORTED;
  const int maxit = S->opts.max_iters > 0 ? S->opts.max_iters : nswp;
  const double tol = S->opts.tol > 0 ? S->opts.tol : 1e-3;
  const int norm = S->opts.norm == 2 ? 2 : 1;
  const bool legacy = nsolv != 3 && nsolv != 4;
  bool refine = S->opts.precision == CMS_PREC_FP32_REFINE;
  LegPlan plan;
  int leg_sweeps = 0;
  if (legacy) {
    if (nsolv >= 6) {
      const int props = legacy_props(S);
      const int kind = legacy_plan(nsolv, nvar, 0.0, maxit, S->opts.nswp0_vel).kind;
      if (!(props & LEG_FIVE_POINT) || (kind == LK_SIP && (!(props & LEG_SIP_ORDER) || !face))) {
        std::snprintf(g_last_error, sizeof(g_last_error),
                      "nsolv %d: SIP, ICCG and ICCGSTAB need four faces per cell, SIP also the natural ordering",
                      nsolv);
        return info->status = CMS_UNSUPPORTED;
      }
    }
    double rm = 0.0;
    if (nsolv == 2 || nsolv == 5) {  // the branch reads this call's rmom
      CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
      CMS_CUDA(cudaStreamSynchronize(S->stream));
      rm = S->h_st->s[S_RMOM];
    }
    plan = legacy_plan(nsolv, nvar, rm, maxit, S->opts.nswp0_vel);
    refine = refine && plan.kind == LK_KRYLOV;  // the hybrid's BiCGStab branch keeps the refinement
  }
  if (plan.kind == LK_NONE) {
  } else if (plan.kind == LK_GS) {
    CHK(run_gauss_seidel<double>(S, S->A64, S->W64, plan.sweeps, plan.symmetric, plan.sor, S->opts.relaxsor,
                                 &leg_sweeps));
  } else if (plan.kind == LK_SIP) {
    CHK(run_sip<double>(S, S->A64, S->W64, face, maxit, nD));
  } else if (plan.kind == LK_ICCG) {
    CHK(run_iccg<double>(S, S->A64, S->W64, maxit));
  } else if (plan.kind == LK_ICCGSTAB) {
    CHK(run_iccgstab<double>(S, S->A64, S->W64, maxit));
  } else if (refine) {
    CHK(run_refine(S, legacy ? 3 : nsolv, maxit, tol, info));
  } else {
    CHK(run_krylov<double>(S, S->A64, S->W64, legacy ? 3 : nsolv, maxit, norm, tol, 0));
  }
  CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  const DevState& h = *S->h_st;
  info->rmom = h.s[S_RMOM];
  if (plan.kind == LK_GS || plan.kind == LK_NONE) {
    info->iters = info->inner = leg_sweeps;
  } else if (!refine) {
    info->iters = h.iter;
    info->inner = (nsolv == 4) ? h.inner : h.iter;
    info->relres = h.s[S_RELRES];
    if (h.nonfinite) info->status = CMS_NONFINITE;
    else if (!h.converged) info->status = CMS_NOT_CONVERGED;
  }
  return info->status;
}

// Eddy-viscosity recurrence lists (flow_eddyvis.f90:169-209): wet cells with
// a face to a dry cell or a dummy (wall cells), and corner cells.
static bool wall_cell(const FlowGeom& g, int i) {
  if (g.iwet[i] != 1) return false;
  for (int k = 0; k < g.ncface[i]; ++k) {
    const int c = g.nb[(size_t)i * g.nmf + k];
    if (c >= g.n || g.iwet[c] == 0) return true;
  }
  return false;
}

static void vis_membership_full(Flow* F) {
  FlowGeom& g = F->geom;
  const int n = F->n;
  F->wall_mem.assign(n, 0);
  F->wall_list.clear();
  F->corner_list.clear();
  for (int i = 0; i < n; ++i) {
    if (wall_cell(g, i)) { F->wall_mem[i] = 1; F->wall_list.push_back(i); }
    if (g.icorner[i]) F->corner_list.push_back(i);
  }
  F->vpos.assign(n, -1);
  F->vlast.assign(n, -1);
}

// Corner flags and list membership of the touched active cells (natural ids).
static void vis_membership_update(Flow* F, const std::vector<int>& touched) {
  FlowGeom& g = F->geom;
  const int nmf = F->nmf;
  std::vector<int> wadd, wdel, cadd, cdel;
  for (int i : touched) {
    int nd = 0;
    if (g.iwet[i] == 1)
      for (int k = 0; k < g.ncface[i]; ++k) nd += (g.iwet[g.nb[(size_t)i * nmf + k]] == 0);
    const int corner = (g.iwet[i] == 1 && nd > 1) ? 1 : 0;
    if (corner != g.icorner[i]) { (corner ? cadd : cdel).push_back(i); g.icorner[i] = corner; }
    const unsigned char w = wall_cell(g, i) ? 1 : 0;
    if (w != F->wall_mem[i]) { (w ? wadd : wdel).push_back(i); F->wall_mem[i] = w; }
  }
  auto merge = [](std::vector<int>& list, std::vector<int>& add, std::vector<int>& del) {
    if (add.empty() && del.empty()) return;
    std::sort(add.begin(), add.end());
    std::sort(del.begin(), del.end());
    std::vector<int> out;
    out.reserve(list.size() + add.size());
    size_t a = 0, d = 0;
    for (int x : list) {
      while (a < add.size() && add[a] < x) out.push_back(add[a++]);
      while (d < del.size() && del[d] < x) ++d;
      if (d < del.size() && del[d] == x) { ++d; continue; }
      out.push_back(x);
    }
    while (a < add.size()) out.push_back(add[a++]);
    list.swap(out);
  };
  merge(F->wall_list, wadd, wdel);
  merge(F->corner_list, cadd, cdel);
}

// Level schedules of the two recurrences from the lists (work in the list
// sizes): a cell is placed after every earlier list cell whose update it reads.
// Wall cells (kf_vis_wall): reads of earlier list cells are marked in rd_cur;
// a read of a dry active cell takes the value of the last earlier list cell
// that wrote it (src, a face of d_wallv), and the dry cells written get their
// last writer's value afterwards (kf_vis_wall_final).  Corner cells
// (kf_vis_corner): reads of earlier corner cells are marked in rd_cur.
static int vis_schedules(Flow* F) {
  const FlowGeom& g = F->geom;
  const int n = F->n, nD = F->nD, nmf = F->nmf;
  static const int kk_of[5] = {0, 3, 4, 1, 2};
  auto nbf = [&](int i, int k) { return g.nb[(size_t)i * nmf + k]; };
  auto drf = [&](int i, int k) { return g.dir[(size_t)i * nmf + k]; };
  auto wallface = [&](int i, int k) { const int c = nbf(i, k); return c >= n || g.iwet[c] == 0; };
  std::vector<int>& pos = F->vpos;
  std::vector<int>& lastw = F->vlast;
  cudaStream_t s = F->S->stream;
  // wall cells
  const std::vector<int>& wl = F->wall_list;
  const int m = (int)wl.size();
  std::vector<int> level(m, 0), src((size_t)m * nmf, -1), written;
  std::vector<unsigned char> cur(m, 0);
  for (int p = 0; p < m; ++p) pos[wl[p]] = p;
  for (int p = 0; p < m; ++p) {
    const int i = wl[p];
    int l = 0;
    for (int k = 0; k < g.ncface[i]; ++k) {
      if (!wallface(i, k)) continue;
      const int kkdf = kk_of[drf(i, k)];
      for (int kk = 0; kk < g.ncface[i]; ++kk) {
        if (drf(i, kk) != kkdf) continue;
        const int c = nbf(i, kk);
        if (c >= n) continue;
        if (g.iwet[c] == 0) {
          const int w = lastw[c];  // earlier list cells only: i's own writes are noted below
          src[(size_t)p * nmf + kk] = w;
          if (w >= 0) l = std::max(l, level[w / nmf] + 1);
        } else if (pos[c] >= 0 && pos[c] < p) {
          cur[p] |= (unsigned char)(1u << kk);
          l = std::max(l, level[pos[c]] + 1);
        }
      }
    }
    level[p] = l;
    for (int k = 0; k < g.ncface[i]; ++k) {
      const int c = nbf(i, k);
      if (c < n && g.iwet[c] == 0) {
        if (lastw[c] < 0) written.push_back(c);
        lastw[c] = p * nmf + k;
      }
    }
  }
  int L = 0;
  for (int p = 0; p < m; ++p) L = std::max(L, level[p] + 1);
  F->wall_lvl.assign(L + 1, 0);
  for (int p = 0; p < m; ++p) F->wall_lvl[level[p] + 1]++;
  for (int l = 0; l < L; ++l) F->wall_lvl[l + 1] += F->wall_lvl[l];
  std::vector<int> fill(F->wall_lvl.begin(), F->wall_lvl.end() - 1), cells(m), srcd((size_t)m * nmf, -1);
  std::vector<unsigned char> rd(m);
  auto face_dev = [&](int w) { return (w % nmf) * nD + F->n2d[wl[w / nmf]]; };
  for (int p = 0; p < m; ++p) {
    const int q = fill[level[p]]++;
    cells[q] = F->n2d[wl[p]];
    rd[q] = cur[p];
    for (int kk = 0; kk < nmf; ++kk) {
      const int w = src[(size_t)p * nmf + kk];
      if (w >= 0) srcd[(size_t)q * nmf + kk] = face_dev(w);
    }
  }
  std::vector<int> fin_c, fin_f;
  std::sort(written.begin(), written.end());
  for (int c : written) { fin_c.push_back(F->n2d[c]); fin_f.push_back(face_dev(lastw[c])); lastw[c] = -1; }
  for (int p = 0; p < m; ++p) pos[wl[p]] = -1;
  F->nwall_fin = (int)fin_c.size();
  if (m > 0) {
    CMS_CUDA(cudaMemcpyAsync(F->d_wall_cells, cells.data(), m * sizeof(int), cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaMemcpyAsync(F->d_wall_rd, rd.data(), m, cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaMemcpyAsync(F->d_wall_src, srcd.data(), srcd.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  }
  if (F->nwall_fin > 0) {
    CMS_CUDA(cudaMemcpyAsync(F->d_wall_fin_cells, fin_c.data(), fin_c.size() * sizeof(int), cudaMemcpyHostToDevice,
                             s));
    CMS_CUDA(cudaMemcpyAsync(F->d_wall_fin_faces, fin_f.data(), fin_f.size() * sizeof(int), cudaMemcpyHostToDevice,
                             s));
  }
  // corner cells
  const std::vector<int>& cl = F->corner_list;
  const int mc = (int)cl.size();
  std::vector<int> clev(mc, 0);
  std::vector<unsigned char> ccur(mc, 0);
  for (int p = 0; p < mc; ++p) pos[cl[p]] = p;
  int LC = 0;
  for (int p = 0; p < mc; ++p) {
    const int i = cl[p];
    int l = 0;
    for (int k = 0; k < g.ncface[i]; ++k) {
      const int c = nbf(i, k);
      if (c < n && pos[c] >= 0 && pos[c] < p) {
        ccur[p] |= (unsigned char)(1u << k);
        l = std::max(l, clev[pos[c]] + 1);
      }
    }
    clev[p] = l;
    LC = std::max(LC, l + 1);
  }
  for (int p = 0; p < mc; ++p) pos[cl[p]] = -1;
  F->corner_lvl.assign(LC + 1, 0);
  for (int p = 0; p < mc; ++p) F->corner_lvl[clev[p] + 1]++;
  for (int l = 0; l < LC; ++l) F->corner_lvl[l + 1] += F->corner_lvl[l];
  std::vector<int> cfill(F->corner_lvl.begin(), F->corner_lvl.end() - 1), ccells(mc);
  std::vector<unsigned char> crd(mc);
  for (int p = 0; p < mc; ++p) {
    const int q = cfill[clev[p]]++;
    ccells[q] = F->n2d[cl[p]];
    crd[q] = ccur[p];
  }
  if (mc > 0) {
    CMS_CUDA(cudaMemcpyAsync(F->d_corner_cells, ccells.data(), mc * sizeof(int), cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaMemcpyAsync(F->d_corner_rd, crd.data(), mc, cudaMemcpyHostToDevice, s));
  }
  CMS_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
  return CMS_OK;
}

// The host wet flags (natural order) into the device copy.
static int wet_upload(Flow* F) {
  std::vector<int> w(F->nD);
  for (int r = 0; r < F->nD; ++r) w[r] = F->geom.iwet[F->d2n[r]];
  CMS_CUDA(cudaMemcpyAsync(F->d_iwet, w.data(), w.size() * sizeof(int), cudaMemcpyHostToDevice, F->S->stream));
  CMS_CUDA(cudaStreamSynchronize(F->S->stream));
  return CMS_OK;
}

static int flow_create(int ncells, int ncellsD, int nmf, const int* c2c, const int* ncface, const int* idirface,
                       const double* x, const double* y, const double* dx, const double* dy, const double* zb,
                       const double* coefman, int nth, const int* th_cells, const int* th_faces,
                       const cms_flow_opts* opts, Flow** out) {
  if (!out || !c2c || !ncface || !idirface || !x || !y || !dx || !dy || !zb || !coefman || nth < 0 ||
      (nth > 0 && (!th_cells || !th_faces)))
    return CMS_BAD_ARGUMENT;
  auto* F = new Flow();
  cms_flow_default_opts(&F->opts);
  if (opts) F->opts = *opts;
  F->n = ncells; F->nD = ncellsD; F->nmf = nmf;
  auto fail = [&](int rc) { cms_flow_destroy(F); return rc; };
  if (F->opts.ndsch < 0 || F->opts.ndsch > 4) {
    std::snprintf(g_last_error, sizeof(g_last_error),
                  "ADVECTION_SCHEME %d: only the first-order schemes 0-4 (NONE, UPWIND, HYBRID, POWERLAW, "
                  "EXPONENTIAL) are served", F->opts.ndsch);
    return fail(CMS_UNSUPPORTED);
  }
  // wet set: active cells and string dummies wet, other dummies are walls
  std::vector<int> iwet(ncellsD, 0);
  for (int i = 0; i < ncells; ++i) iwet[i] = 1;
  std::vector<unsigned char> thm(ncellsD, 0);
  for (int j = 0; j < nth; ++j) {
    const int i = th_cells[j] - 1, k = th_faces[j] - 1;
    if (i < 0 || i >= ncells || k < 0 || k >= nmf) return fail(CMS_BAD_ARGUMENT);
    const int g = c2c[(size_t)i * nmf + k] - 1;
    if (g < ncells || g >= ncellsD) return fail(CMS_BAD_ARGUMENT);
    if (thm[i] & (1u << k)) return fail(CMS_BAD_ARGUMENT);
    thm[i] |= (unsigned char)(1u << k);
    iwet[g] = 1;
  }
  std::string err = build_flow_geom(ncells, ncellsD, nmf, c2c, ncface, idirface, x, y, dx, dy, zb, iwet.data(),
                                    F->opts.skewcor != 0, F->geom);
  if (!err.empty()) {
    std::snprintf(g_last_error, sizeof(g_last_error), "%s", err.c_str());
    return fail(CMS_BAD_ARGUMENT);
  }
  const FlowGeom& g = F->geom;
  const bool skew = F->opts.skewcor && g.njoint > 0;
  F->opts.skewcor = skew ? 1 : 0;
  // solver on the same grid (its device order is the flow's)
  cms_solver_opts so;
  cms_solver_default_opts(&so);
  so.ordering = F->opts.ordering;
  so.precision = F->opts.precision;
  so.tol = F->opts.tol;
  so.norm = F->opts.norm;
  so.verify = 0;
  so.inner_tol = F->opts.inner_tol;
  so.inner_max = F->opts.inner_max;
  so.multi_kernel = F->opts.multi_kernel;
  if (F->opts.relaxsor > 0.0) so.relaxsor = F->opts.relaxsor;
  so.reduced_layout = F->opts.reduced_layout;
  int rc = cms_solver_create(ncells, ncellsD, nmf, c2c, ncface, iwet.data(), &so, &F->S);
  if (rc) return fail(rc);
  Solver* S = F->S;
  const HostPattern& P = S->hp;
  const int n = ncells, nD = ncellsD;
  F->d2n.resize(nD); F->n2d.resize(nD);
  for (int r = 0; r < n; ++r) { F->d2n[r] = P.perm[r]; F->n2d[P.perm[r]] = r; }
  for (int i = n; i < nD; ++i) { F->d2n[i] = i; F->n2d[i] = i; }
  // slot-major face arrays in device order
  auto faceperm_d = [&](const std::vector<double>& a) {
    std::vector<double> o((size_t)nmf * nD, 0.0);
    for (int r = 0; r < nD; ++r)
      for (int k = 0; k < nmf; ++k) o[(size_t)k * nD + r] = a[(size_t)F->d2n[r] * nmf + k];
    return o;
  };
  auto cellperm_d = [&](const std::vector<double>& a) {
    std::vector<double> o(nD, 0.0);
    for (int r = 0; r < nD; ++r) o[r] = a[F->d2n[r]];
    return o;
  };
  std::vector<int> nb((size_t)nmf * nD, -1), ncf(nD);
  std::vector<signed char> back((size_t)nmf * nD, -1), dir((size_t)nmf * nD, 0), fsd((size_t)nmf * n, -1);
  std::vector<unsigned char> owned(nD, 0), thd(nD, 0), joint(nD, 0), crm(nD, 0);
  std::vector<int> iwd(nD);
  for (int r = 0; r < nD; ++r) {
    const int i = F->d2n[r];
    ncf[r] = g.ncface[i];
    iwd[r] = g.iwet[i];
    joint[r] = g.joint[i];
    crm[r] = g.crmask[i];
    thd[r] = thm[i];
    for (int k = 0; k < nmf; ++k) {
      const int j = g.nb[(size_t)i * nmf + k];
      nb[(size_t)k * nD + r] = (k < g.ncface[i] && j >= 0) ? F->n2d[j] : -1;
      back[(size_t)k * nD + r] = (signed char)g.back[(size_t)i * nmf + k];
      dir[(size_t)k * nD + r] = (signed char)g.dir[(size_t)i * nmf + k];
      if (g.owned[(size_t)i * nmf + k]) owned[r] |= (unsigned char)(1u << k);
      if (r < n) fsd[(size_t)k * n + r] = P.fslot[(size_t)i * nmf + k];
    }
  }
  FlowDev& D = F->G;
  D.n = n; D.nD = nD; D.nmf = nmf; D.nsc = g.nsc; D.ider = g.ider;
  // upwind when there is neither turbulent nor constant viscosity
  // (flow.F90:744-746): mturbul is 5 and cviscon 1e-6 here, so the rule never
  // fires and the scheme is the option's
  D.ndsch = F->opts.ndsch;
  int *p_ncf, *p_nb;
  signed char *p_back, *p_dir;
  unsigned char *p_owned, *p_thm, *p_joint, *p_crm;
  if ((rc = F->upload(&p_ncf, ncf)) || (rc = F->upload(&p_nb, nb)) || (rc = F->upload(&F->d_iwet, iwd)) ||
      (rc = F->upload(&p_back, back)) || (rc = F->upload(&p_dir, dir)) || (rc = F->upload(&p_owned, owned)) ||
      (rc = F->upload(&p_thm, thd)) || (rc = F->upload(&p_joint, joint)) || (rc = F->upload(&p_crm, crm)) ||
      (rc = F->upload(&F->d_fslot_dev, fsd)))
    return fail(rc);
  D.ncface = p_ncf; D.nb = p_nb; D.iwet = F->d_iwet; D.back = p_back; D.dir = p_dir; D.owned = p_owned;
  D.thm = p_thm; D.joint = p_joint; D.crmask = p_crm;
  double *p_ds, *p_dn, *p_dsxy, *p_rx, *p_ry, *p_rpx, *p_rpy, *p_fintp, *p_area, *p_zb, *p_man;
  if ((rc = F->upload(&p_ds, faceperm_d(g.ds))) || (rc = F->upload(&p_dn, faceperm_d(g.dn))) ||
      (rc = F->upload(&p_dsxy, faceperm_d(g.dsxy))) || (rc = F->upload(&p_rx, faceperm_d(g.rx))) ||
      (rc = F->upload(&p_ry, faceperm_d(g.ry))) || (rc = F->upload(&p_rpx, faceperm_d(g.rpx))) ||
      (rc = F->upload(&p_rpy, faceperm_d(g.rpy))) || (rc = F->upload(&p_fintp, faceperm_d(g.fintp))) ||
      (rc = F->upload(&p_area, cellperm_d(g.areap))) || (rc = F->upload(&p_zb, cellperm_d(g.zb))))
    return fail(rc);
  {
    std::vector<double> man(nD, 0.0);
    for (int r = 0; r < n; ++r) man[r] = coefman[F->d2n[r]];
    if ((rc = F->upload(&p_man, man))) return fail(rc);
  }
  D.ds = p_ds; D.dn = p_dn; D.dsxy = p_dsxy; D.rx = p_rx; D.ry = p_ry; D.rpx = p_rpx; D.rpy = p_rpy;
  D.fintp = p_fintp; D.areap = p_area; D.zb = p_zb; D.coefman = p_man;
  // wet-cell gradient operator, [q][n] in device numbering (built by kf_gw_rows)
  {
    const size_t nsc = g.nsc;
    GWOut& O = F->gw;
    if ((rc = F->alloc(&O.ncx, n)) || (rc = F->alloc(&O.ncy, n)) || (rc = F->alloc(&O.ngx, n)) ||
        (rc = F->alloc(&O.ngy, n)) || (rc = F->alloc(&O.icx, nsc * n)) || (rc = F->alloc(&O.icy, nsc * n)) ||
        (rc = F->alloc(&O.igx, nsc * n)) || (rc = F->alloc(&O.igy, nsc * n)) || (rc = F->alloc(&O.wcx, nsc * n)) ||
        (rc = F->alloc(&O.wcy, nsc * n)) || (rc = F->alloc(&O.wgxy, nsc * n)) || (rc = F->alloc(&O.wgyx, nsc * n)))
      return fail(rc);
    D.ncx = O.ncx; D.ncy = O.ncy; D.icx = O.icx; D.icy = O.icy; D.ngx = O.ngx; D.ngy = O.ngy; D.igx = O.igx;
    D.igy = O.igy; D.wcx = O.wcx; D.wcy = O.wcy; D.wgxy = O.wgxy; D.wgyx = O.wgyx;
  }
  // wetting and drying: closed dummies (every dummy off the string) and the
  // string's cells and dummies as flow_pond seeds
  {
    WetDryRules& R = F->wd;
    R.closed.assign(nD, 0);
    for (int i = n; i < nD; ++i) R.closed[i] = 1;
    for (int j = 0; j < nth; ++j) {
      const int i = th_cells[j] - 1, k = th_faces[j] - 1;
      const int gd = c2c[(size_t)i * nmf + k] - 1;
      R.closed[gd] = 0;
      R.seed_cells.push_back(i);
      R.seed_dummies.push_back(gd);
    }
    R.ponding = F->opts.ponding != 0;
    R.narrowchannels = F->opts.narrowchannels != 0;
    if ((rc = F->alloc(&F->d_code, nD)) || (rc = F->alloc(&F->d_list, (size_t)n + nD)) ||
        (rc = F->alloc(&F->d_buf, (size_t)3 * nD)) || (rc = F->alloc(&F->d_pn, nD)) || (rc = F->alloc(&F->d_par, n)) ||
        (rc = F->alloc(&F->d_seeded, n)) || (rc = F->alloc(&F->d_fchg, n)) || (rc = F->alloc(&F->d_cnt, 1)) ||
        (rc = F->alloc(&F->d_chg, nD)))
      return fail(rc);
    std::vector<int> sd;
    for (int c : R.seed_cells) sd.push_back(F->n2d[c]);
    F->nseedc = (int)sd.size();
    if ((rc = F->upload(&F->d_seedc, sd))) return fail(rc);
  }
  // parameters (flow.F90:21-168, 684-694, friction.F90:44-49).  hdry1 and
  // hdry2 are read only by the narrow-channel removal rules
  // (flow.F90:1340-1424), which run with narrow channels off, and then
  // flow.F90:686-689 has set them to 5 and 2 hdry whatever the
  // DRYING_DEPTH_ONE_CELL/TWO_CELL cards said; with narrow channels on they
  // are not read (flow.F90:1324-1338).
  const double hdry = F->opts.hdry > 0.0 ? F->opts.hdry : 0.05;
  D.grav = 9.81; D.gravinv = 1.0 / 9.81; D.hmin = hdry; D.hdry = hdry; D.hdry1 = 5.0 * hdry; D.hdry2 = 2.0 * hdry;
  D.relax_uv = 0.8; D.relax_p = 1.0;
  D.facpp = 0.2; D.cviscon = 1.0e-6; D.cvisbot = 0.0667; D.cvismax = 20.0; D.wallfac = 1.0;
  D.cvishor2areaavg = 0.2 * 0.2 * g.areaavg;
  // state
  FlowState& T = F->st;
  double** cellarrs[] = {&T.p, &T.h, &T.u, &T.v, &T.pp, &T.vis, &T.vis0, &T.vis1, &T.cfrict, &T.z0, &T.uv,
                         &T.bsvel, &T.eta, &T.u1, &T.v1, &T.p1, &T.h1, &T.su, &T.sv, &T.sp, &T.spu, &T.spv,
                         &T.ssu0, &T.ssv0, &T.spuv0, &T.sppp0, &T.sspp0, &T.apuareap, &T.sumu, &T.Hu, &T.Hv, &T.res};
  for (double** a : cellarrs)
    if ((rc = F->alloc(a, nD))) return fail(rc);
  double** facearrs[] = {&T.flux, &T.visk, &T.hk, &T.pk, &T.acoef, &T.zbk};
  for (double** a : facearrs)
    if ((rc = F->alloc(a, (size_t)nmf * nD))) return fail(rc);
  for (int c = 0; c < 2; ++c) {
    double** g2[] = {&T.dpx[c], &T.dpy[c], &T.dux[c], &T.duy[c], &T.dvx[c], &T.dvy[c], &T.dppx[c], &T.dppy[c],
                     &T.dHux[c], &T.dHuy[c], &T.dHvx[c], &T.dHvy[c], &T.dapx[c], &T.dapy[c], &T.dzbx[c], &T.dzby[c]};
    for (double** a : g2)
      if ((rc = F->alloc(a, nD))) return fail(rc);
  }
  if ((rc = F->alloc(&T.wsebnd, std::max(nth, 1))) || (rc = F->alloc(&T.flag, 4))) return fail(rc);
  T.chg = F->d_chg;
  if ((rc = F->alloc(&F->d_wse_cell, nD))) return fail(rc);
  F->d_wse = T.wsebnd;
  if (cudaMallocHost((void**)&F->h_flag, 4 * sizeof(int)) != cudaSuccess) return fail(CMS_DEVICE_ERROR);
  // strings
  {
    F->nth = nth;
    std::vector<int> tc(nth), tg(nth);
    for (int j = 0; j < nth; ++j) {
      const int i = th_cells[j] - 1, k = th_faces[j] - 1;
      tc[j] = F->n2d[i];
      tg[j] = F->n2d[c2c[(size_t)i * nmf + k] - 1];
      F->th_cell_nat.push_back(i);
      F->th_dummy_nat.push_back(c2c[(size_t)i * nmf + k] - 1);
    }
    if ((rc = F->upload(&F->d_th_cell, tc)) || (rc = F->upload(&F->d_th_dummy, tg))) return fail(rc);
    std::vector<int> wc, wg;
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < g.ncface[i]; ++k) {
        const int j = g.nb[(size_t)i * nmf + k];
        if (j >= n && !(thm[i] & (1u << k))) { wc.push_back(F->n2d[i]); wg.push_back(F->n2d[j]); }
      }
    F->nw = (int)wc.size();
    if ((rc = F->upload(&F->d_w_cell, wc)) || (rc = F->upload(&F->d_w_dummy, wg))) return fail(rc);
  }
  // eddy-viscosity recurrences next to dry/dummy neighbours and at corners
  if ((rc = F->alloc(&F->d_wall_cells, n)) || (rc = F->alloc(&F->d_wall_rd, n)) ||
      (rc = F->alloc(&F->d_wall_src, (size_t)n * nmf)) || (rc = F->alloc(&F->d_wallv, (size_t)nmf * nD)) ||
      (rc = F->alloc(&F->d_wall_fin_cells, n)) || (rc = F->alloc(&F->d_wall_fin_faces, n)) ||
      (rc = F->alloc(&F->d_corner_cells, n)) || (rc = F->alloc(&F->d_corner_rd, n)))
    return fail(rc);
  vis_membership_full(F);
  if ((rc = vis_schedules(F))) return fail(rc);
  for (int i = 0; i < n; ++i) F->nfaces += g.ncface[i];
  if (cudaStreamSynchronize(S->stream) != cudaSuccess) return fail(CMS_DEVICE_ERROR);
  *out = F;
  return CMS_OK;
}

static inline int fblk(int m) { return (m + TPB - 1) / TPB; }
// algorithmic bytes of a flow kernel: c cell doubles per active cell, f face
// doubles per face, plus per-dummy-cell doubles d (connectivity included as
// 8 bytes per face read)
static inline double fbytes(const Flow* F, double c, double f, double d = 0.0) {
  return 8.0 * (c * F->n + f * F->nfaces + d * (F->nD - F->n));
}

// gradient into the other copy, reading the current one as "previous"
static int grad1(Flow* F, const double* a, double* const* gx, double* const* gy, int& cur) {
  const int nx = 1 - cur;
  FLAUNCHB(F, fbytes(F, 9, 1.5), (kf_grad<1><<<fblk(F->n), TPB, 0, F->S->stream>>>(F->G, a, nullptr, gx[nx], gy[nx], nullptr, nullptr,
                                                               gx[cur], gy[cur], nullptr, nullptr)));
  cur = nx;
  return CMS_OK;
}
static int grad2(Flow* F, const double* a, const double* b, double* const* ax, double* const* ay, double* const* bx,
                 double* const* by, int& cur) {
  const int nx = 1 - cur;
  FLAUNCHB(F, fbytes(F, 13, 3), (kf_grad<2><<<fblk(F->n), TPB, 0, F->S->stream>>>(F->G, a, b, ax[nx], ay[nx], bx[nx], by[nx], ax[cur],
                                                               ay[cur], bx[cur], by[cur])));
  cur = nx;
  return CMS_OK;
}

// solve(acoef,ss,sp,res,phi,n) on the flow state (device order)
// solve() prologue of one flow system: the device-order system (and its FP32
// copy for refinement) from the face coefficients, and rmom.
static int flow_solve_begin(Flow* F, double* ss, const double* sp, double* phi, double relax) {
  Solver* S = F->S;
  const bool refine = S->opts.precision == CMS_PREC_FP32_REFINE;
  // reduction kernel: its grid must stay within the solver's partials buffer
  FLAUNCHB(F, fbytes(F, 9, 2.6), (kf_solve_prologue<float><<<gsz(F->n), TPB, 0, S->stream>>>(
                 F->G, F->st.acoef, ss, sp, F->st.res, phi, F->d_fslot_dev, relax, S->A64.aoff, S->A64.diag,
                 S->W64.b, S->W64.x, refine ? S->A32.aoff : nullptr, refine ? S->A32.diag : nullptr, S->d_part,
                 S->d_st)));
  return CMS_OK;
}

// The solution back into the flow field.
static int flow_solve_end(Flow* F, double* phi, double* rmom, const cms_solve_info* info) {
  FLAUNCHB(F, fbytes(F, 2, 0), (kf_copy<<<fblk(F->n), TPB, 0, F->S->stream>>>(F->n, F->S->W64.x, phi)));
  *rmom = info->rmom;
  return CMS_OK;
}

static int flow_solve(Flow* F, double* ss, const double* sp, double* phi, double relax, int nswp, double* rmom,
                      cms_solve_info* info) {
  CHK(flow_solve_begin(F, ss, sp, phi, relax));
  const int nvar = phi == F->st.u ? 2 : phi == F->st.v ? 3 : 1;
  const int rc = solve_core64(F->S, F->opts.nsolv, nswp, info, nvar, F->st.acoef, F->nD);
  if (rc == CMS_DEVICE_ERROR || rc == CMS_UNSUPPORTED || rc == CMS_BAD_ARGUMENT) return rc;
  return flow_solve_end(F, phi, rmom, info);
}

// eddy viscosity with the boundary recurrences and its face values
static int flow_vis(Flow* F, const double* dux, const double* duy, const double* dvx, const double* dvy) {
  cudaStream_t s = F->S->stream;
  FLAUNCHB(F, fbytes(F, 15, 0), (kf_fric_vis<<<fblk(F->n), TPB, 0, s>>>(F->G, F->st, dux, duy, dvx, dvy, 1)));
  if (F->nth)
    FLAUNCH(F, (kf_copy_to_dummy<<<fblk(F->nth), TPB, 0, s>>>(F->d_th_cell, F->d_th_dummy, F->nth, F->st.vis)));
  FLAUNCHB(F, fbytes(F, 2, 0, 2), (kf_copy<<<fblk(F->nD), TPB, 0, s>>>(F->nD, F->st.vis, F->st.vis0)));
  for (size_t l = 0; l + 1 < F->wall_lvl.size(); ++l) {
    const int a = F->wall_lvl[l], m = F->wall_lvl[l + 1] - a;
    FLAUNCH(F, (kf_vis_wall<<<fblk(m), TPB, 0, s>>>(F->G, F->st, F->d_wall_cells + a, F->d_wall_rd + a,
                                                     F->d_wall_src + (size_t)a * F->nmf, F->d_wallv, m)));
  }
  if (F->nwall_fin)
    FLAUNCH(F, (kf_vis_wall_final<<<fblk(F->nwall_fin), TPB, 0, s>>>(F->d_wall_fin_cells, F->d_wall_fin_faces,
                                                                     F->nwall_fin, F->d_wallv, F->st.vis)));
  FLAUNCHB(F, fbytes(F, 2, 0, 2), (kf_copy<<<fblk(F->nD), TPB, 0, s>>>(F->nD, F->st.vis, F->st.vis1)));
  for (size_t l = 0; l + 1 < F->corner_lvl.size(); ++l) {
    const int a = F->corner_lvl[l], m = F->corner_lvl[l + 1] - a;
    FLAUNCH(F, (kf_vis_corner<<<fblk(m), TPB, 0, s>>>(F->G, F->st, F->d_corner_cells + a, F->d_corner_rd + a, m)));
  }
  FLAUNCHB(F, fbytes(F, 2, 2.5), (kf_interp<<<fblk(F->n), TPB, 0, s>>>(F->G, F->st.vis, 3, F->st.visk, nullptr, nullptr)));
  return CMS_OK;
}

// flow_grad_interp: velocity gradients, face pressure, dp/dx, dp/dy, hk
static int flow_grad_interp(Flow* F) {
  FlowState& T = F->st;
  cudaStream_t s = F->S->stream;
  FCHK(grad2(F, T.u, T.v, T.dux, T.duy, T.dvx, T.dvy, F->cur_duv));
  const bool skew = F->opts.skewcor != 0;
  FLAUNCHB(F, fbytes(F, 4, 2.5), (kf_interp<<<fblk(F->n), TPB, 0, s>>>(F->G, T.p, 1, T.pk, skew ? T.dpx[0] : nullptr,
                                                     skew ? T.dpy[0] : nullptr)));
  FLAUNCHB(F, fbytes(F, 3, 4.2), (kf_dp_hk<<<fblk(F->n), TPB, 0, s>>>(F->G, T, T.dpx[0], T.dpy[0])));
  return CMS_OK;
}

// Wet-cell gradient operator of the listed cells (device numbering), or of
// every active cell when cells is null.
static int gw_rows(Flow* F, const std::vector<int>* cells) {
  cudaStream_t s = F->S->stream;
  if (!cells) {
    FLAUNCH(F, (kf_gw_rows<<<fblk(F->n), TPB, 0, s>>>(F->G, F->gw, nullptr, F->n)));
    return CMS_OK;
  }
  const int m = (int)cells->size();
  if (m == 0) return CMS_OK;
  CMS_CUDA(cudaMemcpyAsync(F->d_list, cells->data(), m * sizeof(int), cudaMemcpyHostToDevice, s));
  FLAUNCH(F, (kf_gw_rows<<<fblk(m), TPB, 0, s>>>(F->G, F->gw, F->d_list, m)));
  CMS_CUDA(cudaStreamSynchronize(s));  // d_list is reused
  return CMS_OK;
}

// Cold-start wet set (natural order, all nD cells): device flags, corner
// flags, eddy-viscosity lists and the whole wet-cell gradient operator
// (der_init builds it from the wet set of flow_init's flow_wetdry call).
static int wetdry_cold(Flow* F, const std::vector<int>& neww) {
  FlowGeom& g = F->geom;
  g.iwet = neww;
  int nwet = 0;
  for (int i = 0; i < F->n; ++i) nwet += neww[i];
  F->nwet = nwet;
  F->last_changed = 0;
  corner_flags(g);
  vis_membership_full(F);
  FCHK(vis_schedules(F));
  FCHK(wet_upload(F));
  return gw_rows(F, nullptr);
}

// The rest of flow_wetdry(0) and der_update after the final wet flags of the
// active cells in act (natural ids; the device flags already hold them) and
// of the dummies in dum (natural ids, new flags in pn) changed
// (flow.F90:1460-1524, derivatives.f90:204-296): corner flags and recurrence
// lists around the changes, dry-to-wet initialisation of u, v, vis (5 passes
// in cell order over the newly wet cells, on a gathered neighbourhood), zero
// flux and viscosity on the faces of cells that became dry, and the gradient
// operator rows of every changed active cell and its neighbours.
static int wetdry_apply(Flow* F, std::vector<int>& act, const std::vector<int>& dum) {
  FlowGeom& g = F->geom;
  const int n = F->n, nmf = F->nmf;
  cudaStream_t s = F->S->stream;
  if ((int)F->nsc.mark.size() != F->nD) F->nsc.mark.assign(F->nD, 0);
  std::sort(act.begin(), act.end());
  std::vector<int> newly, dried;
  for (int x : act) {
    g.iwet[x] ^= 1;
    (g.iwet[x] ? newly : dried).push_back(x);
    F->nwet += g.iwet[x] ? 1 : -1;
  }
  F->last_changed = (int)act.size();
  std::vector<int> parents;  // cells of changed dummies
  if (!dum.empty()) {
    std::vector<int> idx, val;
    for (int x : dum) {
      g.iwet[x] = F->pn[x];
      idx.push_back(F->n2d[x]);
      val.push_back(g.iwet[x]);
      for (int k = 0; k < g.ncface[x]; ++k) {
        const int c = g.nb[(size_t)x * nmf + k];
        if (c >= 0 && c < n) parents.push_back(c);
      }
    }
    const int m = (int)idx.size();
    CMS_CUDA(cudaMemcpyAsync(F->d_list, idx.data(), m * sizeof(int), cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaMemcpyAsync(F->d_list + m, val.data(), m * sizeof(int), cudaMemcpyHostToDevice, s));
    FLAUNCH(F, (kf_scatter_i32<<<fblk(m), TPB, 0, s>>>(F->d_list, F->d_list + m, m, F->d_iwet)));
    CMS_CUDA(cudaStreamSynchronize(s));
  }
  if (act.empty() && dum.empty()) return CMS_OK;
  // corner flags and recurrence lists of the cells within one face of a change
  {
    std::vector<int> touched;
    std::vector<unsigned char>& mk = F->nsc.mark;
    auto touch = [&](int c) { if (c >= 0 && c < n && !mk[c]) { mk[c] = 1; touched.push_back(c); } };
    for (int x : act) {
      touch(x);
      for (int k = 0; k < g.ncface[x]; ++k) touch(g.nb[(size_t)x * nmf + k]);
    }
    for (int c : parents) touch(c);
    for (int c : touched) mk[c] = 0;
    vis_membership_update(F, touched);
    FCHK(vis_schedules(F));
  }
  // dry-to-wet initialisation on the host from the gathered neighbourhood
  if (!newly.empty()) {
    std::vector<int> pos_list, gat;
    std::vector<int>& pos = F->vpos;
    auto add = [&](int c) {
      if (c < n) {
        if (pos[c] < 0) { pos[c] = (int)gat.size(); gat.push_back(c); }
      } else {
        for (size_t q = 0; q < gat.size(); ++q)
          if (gat[q] == c) return;
        gat.push_back(c);
      }
    };
    for (int i : newly) {
      add(i);
      for (int k = 0; k < g.ncface[i]; ++k) add(g.nb[(size_t)i * nmf + k]);
    }
    auto where = [&](int c) -> int {
      if (c < n) return pos[c];
      for (size_t q = 0; q < gat.size(); ++q)
        if (gat[q] == c) return (int)q;
      return -1;
    };
    const int m = (int)gat.size();
    std::vector<int> gdev(m);
    for (int q = 0; q < m; ++q) gdev[q] = F->n2d[gat[q]];
    std::vector<double> buf((size_t)3 * m);
    CMS_CUDA(cudaMemcpyAsync(F->d_list, gdev.data(), m * sizeof(int), cudaMemcpyHostToDevice, s));
    FLAUNCH(F, (kf_gather_uvv<<<fblk(m), TPB, 0, s>>>(F->d_list, m, F->st.u, F->st.v, F->st.vis, F->d_buf)));
    CMS_CUDA(cudaMemcpyAsync(buf.data(), F->d_buf, buf.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CMS_CUDA(cudaStreamSynchronize(s));
    const double small = 1.0e-15;  // definitions.F90:93
    for (int pass = 0; pass < 5; ++pass)
      for (int i : newly) {
        double us = 0.0, vs = 0.0, viss = 0.0;
        int ns = 0;
        for (int k = 0; k < g.ncface[i]; ++k) {
          const int c = g.nb[(size_t)i * nmf + k], q = where(c);
          us = us + buf[3 * q]; vs = vs + buf[3 * q + 1]; viss = viss + buf[3 * q + 2];
          ns += g.iwet[c];
        }
        const int q = pos[i];
        buf[3 * q] = us / ((double)ns + small) / 1.25;
        buf[3 * q + 1] = vs / ((double)ns + small) / 1.25;
        buf[3 * q + 2] = viss / ((double)ns + small);
      }
    const int mn = (int)newly.size();
    std::vector<double> out((size_t)3 * mn);
    for (int j = 0; j < mn; ++j) {
      const int q = pos[newly[j]];
      gdev[j] = F->n2d[newly[j]];
      for (int c = 0; c < 3; ++c) out[3 * j + c] = buf[3 * q + c];
    }
    for (int c : gat)
      if (c < n) pos[c] = -1;
    CMS_CUDA(cudaMemcpyAsync(F->d_list, gdev.data(), mn * sizeof(int), cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaMemcpyAsync(F->d_buf, out.data(), out.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    FLAUNCH(F, (kf_scatter_uvv<<<fblk(mn), TPB, 0, s>>>(F->d_list, mn, F->d_buf, F->st.u, F->st.v, F->st.vis)));
    CMS_CUDA(cudaStreamSynchronize(s));
  }
  // faces of the cells that became dry, and of the cells of dummies that did
  {
    std::vector<int> zl;
    for (int x : dried) zl.push_back(F->n2d[x]);
    for (int c : parents) zl.push_back(F->n2d[c]);
    if (!zl.empty()) {
      const int m = (int)zl.size();
      CMS_CUDA(cudaMemcpyAsync(F->d_list, zl.data(), m * sizeof(int), cudaMemcpyHostToDevice, s));
      FLAUNCH(F, (kf_wet_faces_list<<<fblk(m), TPB, 0, s>>>(F->G, F->st, F->d_list, m)));
      CMS_CUDA(cudaStreamSynchronize(s));
    }
  }
  // der_update's list: changed active cells and their active neighbours
  if (act.empty()) return CMS_OK;
  std::vector<int> list;
  std::vector<unsigned char>& mk = F->nsc.mark;
  auto mark = [&](int c) { if (c >= 0 && c < n && !mk[c]) { mk[c] = 1; list.push_back(c); } };
  for (int x : act) {
    mark(x);
    for (int k = 0; k < g.ncface[x]; ++k) mark(g.nb[(size_t)x * nmf + k]);
  }
  for (int& c : list) { mk[c] = 0; c = F->n2d[c]; }
  return gw_rows(F, &list);
}

// Wet/dry update at the start of a step whose depth classes changed: the
// changed classes come back as a list, the narrow-channel set is updated
// incrementally on the host, flow_pond runs on the device (union-find over
// the new narrow-channel set), and the changes of the final flags are
// applied (wetdry_apply).
static int wetdry_update(Flow* F, int nchg) {
  using clk = std::chrono::steady_clock;
  auto ms = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
  const auto t0 = clk::now();
  const int n = F->n;
  cudaStream_t s = F->S->stream;
  std::vector<int> enc(nchg), changed;
  if (nchg > 0) {
    CMS_CUDA(cudaMemcpyAsync(enc.data(), F->d_chg, nchg * sizeof(int), cudaMemcpyDeviceToHost, s));
    CMS_CUDA(cudaStreamSynchronize(s));
  }
  for (int e : enc) {
    const int x = F->d2n[e & 0x0fffffff];
    F->code_nat[x] = (unsigned char)((unsigned)e >> 28);
    changed.push_back(x);
  }
  const auto t1 = clk::now();
  std::vector<int> pch;
  narrow_update(F->geom, F->code_nat.data(), F->wd, changed, F->w0, F->pn, F->nsc, pch);
  const auto t2 = clk::now();
  F->wd_updates++;
  std::vector<int> act, dum;
  std::vector<int> idx;
  std::vector<unsigned char> val;
  for (int x : pch) {
    if (x >= n) {
      if (F->geom.iwet[x] != F->pn[x]) dum.push_back(x);
      continue;
    }
    idx.push_back(F->n2d[x]);
    val.push_back(F->pn[x]);
  }
  if (!idx.empty()) {  // the active part of the narrow-channel set changed: flow_pond again
    const int m = (int)idx.size();
    CMS_CUDA(cudaMemcpyAsync(F->d_list, idx.data(), m * sizeof(int), cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaMemcpyAsync(F->d_buf, val.data(), m, cudaMemcpyHostToDevice, s));
    FLAUNCH(F, (kf_scatter_u8<<<fblk(m), TPB, 0, s>>>(F->d_list, (const unsigned char*)F->d_buf, m, F->d_pn)));
    CMS_CUDA(cudaMemsetAsync(F->d_cnt, 0, sizeof(int), s));
    const int ponding = F->wd.ponding ? 1 : 0;
    if (!ponding) {
      FLAUNCH(F, (kf_pond_init<<<fblk(n), TPB, 0, s>>>(n, F->d_par)));
      FLAUNCH(F, (kf_pond_hook<<<fblk(n), TPB, 0, s>>>(F->G, F->d_pn, F->d_par)));
      CMS_CUDA(cudaMemsetAsync(F->d_seeded, 0, n, s));
      if (F->nseedc)
        FLAUNCH(F, (kf_pond_seed<<<fblk(F->nseedc), TPB, 0, s>>>(F->d_seedc, F->nseedc, F->d_pn, F->d_par,
                                                               F->d_seeded)));
    }
    FLAUNCH(F, (kf_pond_final<<<fblk(n), TPB, 0, s>>>(n, F->d_pn, F->d_par, F->d_seeded, ponding, F->d_iwet,
                                                      F->d_fchg, F->d_cnt)));
    int m2 = 0;
    CMS_CUDA(cudaMemcpyAsync(&m2, F->d_cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    CMS_CUDA(cudaStreamSynchronize(s));
    if (m2 > 0) {
      act.resize(m2);
      CMS_CUDA(cudaMemcpyAsync(act.data(), F->d_fchg, m2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      CMS_CUDA(cudaStreamSynchronize(s));
      for (int& r : act) r = F->d2n[r];
    }
  }
  const int rc = wetdry_apply(F, act, dum);
  const auto t3 = clk::now();
  F->wd_ms[0] += ms(t0, t1); F->wd_ms[1] += ms(t1, t2); F->wd_ms[2] += ms(t2, t3);
  return rc;
}

// Cold start (u_nat == nullptr: at rest) or hot start from the water pressure
// p_nat and velocities u_nat, v_nat of all nD cells (natural order), and the
// face fluxes flux_nat ([nD][nmf]) when the hot-start file holds them.
static int flow_start(Flow* F, std::vector<double> p_nat, const double* u_nat, const double* v_nat,
                      const double* flux_nat = nullptr) {
  FlowState& T = F->st;
  cudaStream_t s = F->S->stream;
  const int nD = F->nD;
  const bool hot = u_nat != nullptr;
  ++F->graph_gen;  // a new wet set and its recurrence lists
  std::vector<double> u0, v0;
  std::vector<int> wet_hot;
  if (hot) {
    // hot_init (hot_start.F90:1164-1200): cells with h < hmin + 1e-5 are dry
    // and at rest; each water-level string dummy takes its cell's values
    u0.assign(u_nat, u_nat + nD);
    v0.assign(v_nat, v_nat + nD);
    wet_hot.assign(nD, 1);
    for (int i = 0; i < nD; ++i) {
      const double hh = p_nat[i] * F->G.gravinv - F->geom.zb[i];
      if (hh < F->G.hmin + 1.0e-5) { wet_hot[i] = 0; u0[i] = v0[i] = 0.0; }
    }
    for (size_t j = 0; j < F->th_cell_nat.size(); ++j) {
      const int i = F->th_cell_nat[j], d = F->th_dummy_nat[j];
      u0[d] = u0[i]; v0[d] = v0[i]; p_nat[d] = p_nat[i];
    }
  }
  // wet set of the cold start (prestart.f90:308-315): flow_wetdry(0), again
  // with ponding on when every cell is dry
  {
    std::vector<unsigned char>& cn = F->code_nat;
    cn.assign(nD, 0);
    for (int i = 0; i < nD; ++i) {
      const double pi = p_nat[i];
      const double hh = pi * F->G.gravinv - F->geom.zb[i];
      cn[i] = (unsigned char)((hh >= F->G.hdry ? WD_WET : 0) | (hh < F->G.hdry1 ? WD_LT1 : 0) |
                              (hh < F->G.hdry2 ? WD_LT2 : 0));
    }
    std::vector<int> neww;
    depth_set(F->geom, cn.data(), F->wd, F->w0);
    narrow_full(F->geom, cn.data(), F->wd, F->w0, F->pn);
    pond_host(F->geom, F->wd, F->pn, neww);
    int nwet = 0;
    for (int i = 0; i < F->n; ++i) nwet += neww[i];
    if (nwet == 0 && !F->wd.ponding) {
      F->wd.ponding = true;
      pond_host(F->geom, F->wd, F->pn, neww);
    }
    F->nsc = NarrowScratch();
    FCHK(wetdry_cold(F, neww));
    std::vector<unsigned char> cd(nD), pd(nD);
    for (int r = 0; r < nD; ++r) { cd[r] = cn[F->d2n[r]]; pd[r] = F->pn[F->d2n[r]]; }
    CMS_CUDA(cudaMemcpyAsync(F->d_code, cd.data(), nD, cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaMemcpyAsync(F->d_pn, pd.data(), nD, cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaStreamSynchronize(s));
    F->wd_pending = 0;
    F->nchg_pending = 0;
  }
  if (hot) {
    // flow_wetdry(0) against hot_init's wet set: the dry-to-wet initialisation
    // of the cells it wets (flow.F90:1476-1491, five passes in cell order; the
    // viscosities are all zero at this point)
    const FlowGeom& g = F->geom;
    for (int pass = 0; pass < 5; ++pass)
      for (int i = 0; i < F->n; ++i) {
        if (!(g.iwet[i] == 1 && wet_hot[i] == 0)) continue;
        double us = 0.0, vs = 0.0;
        int ns = 0;
        for (int k = 0; k < g.ncface[i]; ++k) {
          const int j = g.nb[(size_t)i * g.nmf + k];
          us = us + u0[j]; vs = vs + v0[j]; ns += g.iwet[j];
        }
        u0[i] = us / ((double)ns + 1.0e-15) / 1.25;
        v0[i] = vs / ((double)ns + 1.0e-15) / 1.25;
      }
  }
  std::vector<double> p(nD), h(nD), eta(nD);
  for (int r = 0; r < nD; ++r) {
    const int i = F->d2n[r];
    p[r] = p_nat[i];
    double hh = p[r] * F->G.gravinv - F->geom.zb[i];
    if (hh < F->G.hdry) hh = std::max(hh, F->G.hmin);
    h[r] = hh;
    eta[r] = F->geom.iwet[i] ? p[r] * F->G.gravinv : -999.0;
  }
  CMS_CUDA(cudaMemcpyAsync(T.p, p.data(), nD * sizeof(double), cudaMemcpyHostToDevice, s));
  CMS_CUDA(cudaMemcpyAsync(T.h, h.data(), nD * sizeof(double), cudaMemcpyHostToDevice, s));
  CMS_CUDA(cudaMemcpyAsync(T.eta, eta.data(), nD * sizeof(double), cudaMemcpyHostToDevice, s));
  const size_t cb = nD * sizeof(double), fb = (size_t)F->nmf * nD * sizeof(double);
  for (double* a : {T.u, T.v, T.pp, T.vis, T.cfrict, T.uv, T.bsvel})
    CMS_CUDA(cudaMemsetAsync(a, 0, cb, s));
  std::vector<double> ud, vd;
  if (hot) {
    ud.resize(nD); vd.resize(nD);
    for (int r = 0; r < nD; ++r) { ud[r] = u0[F->d2n[r]]; vd[r] = v0[F->d2n[r]]; }
    CMS_CUDA(cudaMemcpyAsync(T.u, ud.data(), cb, cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaMemcpyAsync(T.v, vd.data(), cb, cudaMemcpyHostToDevice, s));
  }
  for (double* a : {T.flux, T.visk, T.hk, T.pk, T.acoef, T.zbk}) CMS_CUDA(cudaMemsetAsync(a, 0, fb, s));
  for (int c = 0; c < 2; ++c)
    for (double* a : {T.dpx[c], T.dpy[c], T.dux[c], T.duy[c], T.dvx[c], T.dvy[c], T.dppx[c], T.dppy[c], T.dHux[c],
                      T.dHuy[c], T.dHvx[c], T.dHvy[c], T.dapx[c], T.dapy[c], T.dzbx[c], T.dzby[c]})
      CMS_CUDA(cudaMemsetAsync(a, 0, cb, s));
  F->cur_dppx = F->cur_duv = F->cur_dH = F->cur_dap = 0;
  CMS_CUDA(cudaMemsetAsync(T.flag, 0, 4 * sizeof(int), s));
  // bed slope with the all-cells operator and the face bed elevation (prestart.f90:317-318)
  {
    const FlowGeom& g = F->geom;
    const int n = F->n, nsc = g.nsc;
    std::vector<double> zbr(nD), zx(nD, 0.0), zy(nD, 0.0);
    for (int r = 0; r < nD; ++r) zbr[r] = g.zb[F->d2n[r]];
    for (int i = 0; i < n; ++i) {
      double ax = 0, ay = 0;
      for (int q = 0; q < g.ga_ncx[i]; ++q) ax += g.ga_wcx[(size_t)i * nsc + q] * g.zb[g.ga_icx[(size_t)i * nsc + q]];
      for (int q = 0; q < g.ga_ncy[i]; ++q) ay += g.ga_wcy[(size_t)i * nsc + q] * g.zb[g.ga_icy[(size_t)i * nsc + q]];
      zx[F->n2d[i]] = ax; zy[F->n2d[i]] = ay;
    }
    CMS_CUDA(cudaMemcpyAsync(T.dzbx[0], zx.data(), cb, cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaMemcpyAsync(T.dzby[0], zy.data(), cb, cudaMemcpyHostToDevice, s));
    CMS_CUDA(cudaStreamSynchronize(s));
    FLAUNCH(F, (kf_interp<<<fblk(n), TPB, 0, s>>>(F->G, F->G.zb, 0, T.zbk, F->opts.skewcor ? T.dzbx[0] : nullptr,
                                                  F->opts.skewcor ? T.dzby[0] : nullptr)));
  }
  FCHK(flow_grad_interp(F));
  std::vector<double> fd;
  if (hot && flux_nat) {
    // the file's fluxes, zero across faces flow_wetdry(0) left with a dry side
    // (flow.F90:1497-1512); flow_convflux is skipped (prestart.f90:319)
    const FlowGeom& g = F->geom;
    const int nmf = F->nmf;
    std::vector<double> fn(flux_nat, flux_nat + (size_t)nD * nmf);
    for (int i = 0; i < F->n; ++i)
      for (int k = 0; k < g.ncface[i]; ++k) {
        const size_t f = (size_t)i * nmf + k;
        if (!g.owned[f]) continue;
        const int j = g.nb[f];
        if (g.iwet[i] * g.iwet[j] == 0) { fn[f] = 0.0; fn[(size_t)j * nmf + g.back[f]] = 0.0; }
      }
    fd.assign((size_t)nmf * nD, 0.0);
    for (int i = 0; i < nD; ++i)
      for (int k = 0; k < nmf; ++k) fd[(size_t)k * nD + F->n2d[i]] = fn[(size_t)i * nmf + k];
    CMS_CUDA(cudaMemcpyAsync(T.flux, fd.data(), fb, cudaMemcpyHostToDevice, s));
  } else if (hot) {
    FLAUNCH(F, (kf_convflux<<<fblk(F->n), TPB, 0, s>>>(F->G, T)));
  }
  FCHK(flow_vis(F, T.dux[F->cur_duv], T.duy[F->cur_duv], T.dvx[F->cur_duv], T.dvy[F->cur_duv]));
  CMS_CUDA(cudaStreamSynchronize(s));  // ud, vd are read by the copies above
  // time levels
  FLAUNCH(F, (kf_update<<<fblk(nD), TPB, 0, s>>>(F->G, T, T.dppx[0], T.dppy[0], T.dppx[1], T.dppy[1])));
  CMS_CUDA(cudaStreamSynchronize(s));
  F->t_sim = 0.0;
  F->inited = 1;
  return CMS_OK;
}

// check_conv (flow_imp.F90:1576-1747), dtvar off: 0 divergent, 1 continue, 2 converged
static int check_conv(const double rm[4], double rmom0[4], double rmom1[4], int niter, int maxit) {
  if (niter <= 2)
    for (int q = 1; q <= 3; ++q) { rmom0[q] = std::max(rm[q], 1e-15); rmom1[q] = rmom0[q]; }
  const double rmommax = std::max(rm[1], std::max(rm[2], rm[3]));
  if (rmommax > 5.0) return 0;
  if (niter <= 5) return 1;
  const int nhalf = maxit / 2;
  const double rp = rm[1] / rmom0[1];
  const double ruv = std::max(rm[2] / rmom0[2], rm[3] / rmom0[3]);
  if ((rp >= 0.5 * 10.0 || ruv >= 1.0 * 10.0) && rm[1] > 1e-4) return 0;
  if (niter == maxit && (rp >= 0.5 || ruv >= 1.0) && rm[1] > 1e-3) return 0;
  if (niter == maxit && (rp >= 0.5 / 5.0 || ruv >= 1.0 / 5.0) && rm[1] > 1e-4) return 0;
  const double rmomuv = std::max(rm[2], rm[3]);
  if (rm[1] <= 1e-8 && rmomuv <= 1e-7) return 2;
  if (niter == maxit && (rm[1] > 1e-3 || rmomuv > 1e-2)) return 0;
  if (niter == maxit && (rm[1] > 1e-4 || rmomuv > 1e-3)) return 0;
  if (niter <= nhalf || niter % 2 != 0) return 1;
  const double rchp = rmom1[1] - rm[1];
  const double rchuv = std::max(rmom1[2], rmom1[3]) - rmomuv;
  if (rchp < 0.0 || rchuv < 0.0) return 1;
  if (rchp <= 1e-8 && rchuv <= 1e-7) return 2;
  for (int q = 1; q <= 3; ++q) rmom1[q] = rm[q];
  return 1;
}

// Stages of one time step (flow_imp.F90:29-312), shared by the single-model
// step and the ensemble step.

// before the outer loop: string water levels, static sources
static int step_begin(Flow* F, double dt, const double* wsebnd) {
  FlowState& T = F->st;
  cudaStream_t s = F->S->stream;
  F->last_changed = 0;
  if (F->wd_pending) {  // flow_wetdry(0) and der_update (flow_imp.F90:73-79)
    ++F->graph_gen;     // the recurrence lists may change: stage graphs are captured again
    FCHK(wetdry_update(F, F->nchg_pending));
    F->wd_pending = 0;
    F->nchg_pending = 0;
  }
  if (F->nth) {  // water levels of the string, placed on the string's dummies
    if (wsebnd)
      CMS_CUDA(cudaMemcpyAsync(F->d_wse, wsebnd, F->nth * sizeof(double), cudaMemcpyHostToDevice, s));
    else  // bnd_eval on the device: the constituents at the new time level
      FLAUNCH(F, (kf_tide_eval<<<fblk(F->nth), TPB, 0, s>>>(F->nth, F->ntc, F->d_tide, F->d_psi, F->d_wsevar,
                                                            (F->t_sim + dt) / 3600.0 + F->tide_dtj, F->tide_offset,
                                                            F->d_wse)));
    FLAUNCH(F, (kf_scatter_vals<<<fblk(F->nth), TPB, 0, s>>>(F->d_th_dummy, F->d_wse, F->nth, F->d_wse_cell)));
  }
  FLAUNCHB(F, fbytes(F, 13, 0, 3), (kf_static<<<fblk(F->nD), TPB, 0, s>>>(F->G, T, dt)));
  for (int q = 0; q < 4; ++q) F->it_rm[q] = F->it_rmom0[q] = F->it_rmom1[q] = 0.0;
  F->it_kry = 0;
  std::memset(F->last_solve, 0, 3 * sizeof(cms_solve_info));
  return CMS_OK;
}

static int flow_maxit(const Flow* F) { return F->opts.maxit > 0 ? F->opts.maxit : 20 + F->n / 10000; }

// momentum coefficients (before the u and v solves)
static int stage_uv(Flow* F) {
  FlowState& T = F->st;
  const int cd = F->cur_duv;
  FLAUNCHB(F, fbytes(F, 16.5, 5.6), (kf_coef_uv<<<fblk(F->n), TPB, 0, F->S->stream>>>(F->G, T, T.dux[cd], T.duy[cd],
                                                                                       T.dvx[cd], T.dvy[cd], T.dpx[0],
                                                                                       T.dpy[0])));
  return CMS_OK;
}

// Gradient-copy state of a flow model (the key of its stage graphs).
static inline int stage_key(const Flow* F) { return F->cur_duv | F->cur_dH << 1 | F->cur_dap << 2 | F->cur_dppx << 3; }
static inline void set_stage_key(Flow* F, int k) {
  F->cur_duv = k & 1; F->cur_dH = (k >> 1) & 1; F->cur_dap = (k >> 2) & 1; F->cur_dppx = (k >> 3) & 1;
}

// Runs the kernel sequence fn issues on the solver stream, through a CUDA
// graph when the handle replays graphs: captured on first use for the
// current gradient-copy state (fn's host side -- the copy flips -- runs
// during the capture, so the state after it is recorded and restored on
// every replay), re-captured after a wet-set change.  A capture that fails
// turns graphs off for this handle and runs fn directly.
template <class Fn>
static int run_stage(Flow* F, int which, Fn&& fn) {
  if (!F->use_graphs || F->S->prof_on) return fn();
  cudaStream_t s = F->S->stream;
  const int key = stage_key(F);
  Flow::StageGraph& g = F->sgraph[which][key];
  if (!g.exec || g.gen != F->graph_gen) {
    if (g.exec) {
      cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
    const long long l0 = F->launches;
    cudaGraph_t graph = nullptr;
    int rc = CMS_DEVICE_ERROR;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      rc = fn();
      const cudaError_t e = cudaStreamEndCapture(s, &graph);
      if (e != cudaSuccess) rc = CMS_DEVICE_ERROR;
    }
    if (rc == CMS_OK && graph && cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess) {
      g.exec = nullptr;
      rc = CMS_DEVICE_ERROR;
    }
    if (graph) cudaGraphDestroy(graph);
    if (rc != CMS_OK || !g.exec) {  // nothing ran: undo the host side, launch directly from now on
      cudaGetLastError();
      F->use_graphs = 0;
      F->launches = l0;
      set_stage_key(F, key);
      return fn();
    }
    g.gen = F->graph_gen;
    g.key_after = stage_key(F);
    g.nlaunch = F->launches - l0;
    F->launches = l0;
    ++F->graph_captures;
  }
  CMS_CUDA(cudaGraphLaunch(g.exec, s));
  set_stage_key(F, g.key_after);
  F->launches += g.nlaunch;
  ++F->graph_launches;
  return CMS_OK;
}

// pressure-correction system (after the u and v solves)
static int stage_pp_kernels(Flow* F) {
  FlowState& T = F->st;
  cudaStream_t s = F->S->stream;
  const bool skew = F->opts.skewcor != 0;
  FLAUNCHB(F, fbytes(F, 11.5, 1), (kf_pp_cell<<<fblk(F->n), TPB, 0, s>>>(F->G, T, T.dpx[0], T.dpy[0])));
  if (skew) {
    CHK(grad2(F, T.Hu, T.Hv, T.dHux, T.dHuy, T.dHvx, T.dHvy, F->cur_dH));
    CHK(grad1(F, T.apuareap, T.dapx, T.dapy, F->cur_dap));
  }
  FLAUNCHB(F, fbytes(F, 8, 5), (kf_pp_face<<<fblk(F->n), TPB, 0, s>>>(F->G, T, skew ? 1 : 0, T.dHuy[F->cur_dH],
                                                                     T.dHvx[F->cur_dH], T.dapx[F->cur_dap],
                                                                     T.dapy[F->cur_dap], T.dpx[0], T.dpy[0])));
  FLAUNCHB(F, fbytes(F, 6, 1.2), (kf_pp_src<<<fblk(F->n), TPB, 0, s>>>(F->G, T, skew ? 1 : 0, T.dppx[F->cur_dppx],
                                                                      T.dppy[F->cur_dppx], F->d_wse_cell)));
  return CMS_OK;
}

static int stage_pp(Flow* F) { return run_stage(F, 0, [&] { return stage_pp_kernels(F); }); }

// corrections after the pressure-correction solve
static int stage_corr_kernels(Flow* F) {
  FlowState& T = F->st;
  cudaStream_t s = F->S->stream;
  const bool skew = F->opts.skewcor != 0;
  if (F->nw) FLAUNCH(F, (kf_wall_copy<<<fblk(F->nw), TPB, 0, s>>>(F->d_w_cell, F->d_w_dummy, F->nw, T.pp)));
  CHK(grad1(F, T.pp, T.dppx, T.dppy, F->cur_dppx));
  FLAUNCHB(F, fbytes(F, 9, 2.5), (kf_pvfc<<<fblk(F->n), TPB, 0, s>>>(F->G, T, skew ? 1 : 0, T.dppx[F->cur_dppx],
                                                                    T.dppy[F->cur_dppx])));
  FLAUNCHB(F, fbytes(F, 6, 0, 6), (kf_pvfc_p<<<fblk(F->nD), TPB, 0, s>>>(F->G, T)));
  if (F->nw) FLAUNCH(F, (kf_wall_copy<<<fblk(F->nw), TPB, 0, s>>>(F->d_w_cell, F->d_w_dummy, F->nw, T.p)));
  CHK(flow_grad_interp(F));
  const int c2 = F->cur_duv;
  CHK(flow_vis(F, T.dux[c2], T.duy[c2], T.dvx[c2], T.dvy[c2]));
  return CMS_OK;
}

// corrections, then check_conv
static int stage_corr(Flow* F, int niter, int maxit, int* iconv) {
  CHK(run_stage(F, 1, [&] { return stage_corr_kernels(F); }));
  *iconv = check_conv(F->it_rm, F->it_rmom0, F->it_rmom1, niter, maxit);
  return CMS_OK;
}

// after the outer loop: face velocities and levels, time levels, checks
static int step_end(Flow* F, double dt, int niter, int iconv, cms_flow_info* info) {
  FlowState& T = F->st;
  cudaStream_t s = F->S->stream;
  FLAUNCHB(F, fbytes(F, 8, 3.2), (kf_velface_eta<<<fblk(F->n), TPB, 0, s>>>(F->G, T)));
  FLAUNCH(F, (kf_fric_vis<<<fblk(F->n), TPB, 0, s>>>(F->G, T, nullptr, nullptr, nullptr, nullptr, 0)));
  FLAUNCHB(F, fbytes(F, 13, 0, 13), (kf_update<<<fblk(F->nD), TPB, 0, s>>>(F->G, T, T.dppx[0], T.dppy[0], T.dppx[1],
                                                                           T.dppy[1])));
  FLAUNCH(F, (kf_check<<<fblk(F->n), TPB, 0, s>>>(F->G, T)));
  // depth classes for the next step's flow_wetdry(0) (p does not change in between)
  FLAUNCHB(F, fbytes(F, 0, 0, 0) + 17.0 * F->nD, (kf_wet_codes<<<fblk(F->nD), TPB, 0, s>>>(F->G, T, F->d_code)));
  CMS_CUDA(cudaMemcpyAsync(F->h_flag, T.flag, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
  CMS_CUDA(cudaStreamSynchronize(s));
  if (F->h_flag[2]) {
    F->wd_pending = 1;
    F->nchg_pending = F->h_flag[3];
    CMS_CUDA(cudaMemsetAsync(T.flag + 2, 0, 2 * sizeof(int), s));
  }
  F->t_sim += dt;
  std::memset(info, 0, sizeof(*info));
  info->niter = niter;
  info->iconv = iconv;
  info->rmom_p = F->it_rm[1]; info->rmom_u = F->it_rm[2]; info->rmom_v = F->it_rm[3];
  info->krylov_iters = F->it_kry;
  info->nwet = F->nwet;
  info->nchanged = F->last_changed;
  info->status = CMS_OK;
  if (F->h_flag[1] || iconv == 0) info->status = CMS_NONFINITE;
  F->last = *info;
  return info->status;
}

static int flow_step(Flow* F, double dt, const double* wsebnd, cms_flow_info* info) {
  FlowState& T = F->st;
  cms_flow_info loc{};
  if (!info) info = &loc;
  CHK(step_begin(F, dt, wsebnd));
  const int maxit = flow_maxit(F);
  int iconv = 1, niter = 0;
  cms_solve_info* si = F->last_solve;
  for (niter = 1; niter <= maxit; ++niter) {
    CHK(stage_uv(F));
    std::memset(si, 0, 3 * sizeof(cms_solve_info));
    FCHK(flow_solve(F, T.su, T.spu, T.u, F->G.relax_uv, F->opts.nswp_uv, &F->it_rm[2], &si[0]));
    F->it_kry += si[0].iters;
    if (si[0].status == CMS_NONFINITE) { iconv = 0; break; }
    FCHK(flow_solve(F, T.sv, T.spv, T.v, F->G.relax_uv, F->opts.nswp_uv, &F->it_rm[3], &si[1]));
    F->it_kry += si[1].iters;
    if (si[1].status == CMS_NONFINITE) { iconv = 0; break; }
    CHK(stage_pp(F));
    FCHK(flow_solve(F, T.su, T.sp, T.pp, 1.0, F->opts.nswp_pp, &F->it_rm[1], &si[2]));
    F->it_kry += si[2].iters;
    if (si[2].status == CMS_NONFINITE) { iconv = 0; break; }
    CHK(stage_corr(F, niter, maxit, &iconv));
    if (iconv == 0 || iconv == 2) break;
  }
  if (niter > maxit) niter = maxit;
  return step_end(F, dt, niter, iconv, info);
}

}  // namespace cms

extern "C" {

void cms_flow_default_opts(cms_flow_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->nsolv = 4;
  o->ordering = CMS_ORDER_MULTICOLOR;
  o->precision = CMS_PREC_FP64;
  o->norm = 1;
  o->tol = 1.0e-3;
  o->nswp_pp = 20;
  o->nswp_uv = 5;
  o->maxit = 0;
  o->skewcor = 1;
  o->inner_tol = 0.0;
  o->inner_max = 0;
  o->hdry = 0.05;
  o->ponding = 0;
  o->narrowchannels = 0;
  o->relaxsor = 1.8;
  o->ndsch = 4;
}

int cms_flow_create(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface,
                    const int* idirface, const double* x, const double* y, const double* dx, const double* dy,
                    const double* zb, const double* coefman, int nth, const int* th_cells, const int* th_faces,
                    const cms_flow_opts* opts, cms_flow** out) {
  return cms::flow_create(ncells, ncellsD, nmaxfaces, cell2cell, ncface, idirface, x, y, dx, dy, zb, coefman, nth,
                          th_cells, th_faces, opts, out);
}

int cms_flow_init(cms_flow* f, const double* eta0) {
  if (!f || !eta0) return CMS_BAD_ARGUMENT;
  std::vector<double> p(f->nD);
  for (int i = 0; i < f->nD; ++i) p[i] = eta0[i] * f->G.grav;
  return cms::flow_start(f, std::move(p), nullptr, nullptr);
}

int cms_flow_init_hot(cms_flow* f, const double* p, const double* u, const double* v, const double* flux) {
  if (!f || !p || !u || !v) return CMS_BAD_ARGUMENT;
  return cms::flow_start(f, std::vector<double>(p, p + f->nD), u, v, flux);
}

int cms_flow_step(cms_flow* f, double dt, const double* wsebnd, cms_flow_info* info) {
  if (!f || !f->inited || dt <= 0.0 || (f->nth > 0 && !wsebnd && f->ntc == 0)) return CMS_BAD_ARGUMENT;
  return cms::flow_step(f, dt, wsebnd, info);
}

int cms_flow_set_tide(cms_flow* f, int ntc, const double* amp, const double* speed, const double* phase,
                      const double* nodal, const double* vu, const double* psi, const double* wsevar, double dtj,
                      double offset) {
  if (!f || ntc <= 0 || !amp || !speed || !phase || f->nth <= 0) return CMS_BAD_ARGUMENT;
  const int nth = f->nth;
  std::vector<double> coef((size_t)ntc * 5), ps((size_t)nth * ntc, 0.0), var(nth, 0.0);
  for (int k = 0; k < ntc; ++k) {
    coef[5 * k + 0] = nodal ? nodal[k] : 1.0;
    coef[5 * k + 1] = amp[k];
    coef[5 * k + 2] = speed[k];
    coef[5 * k + 3] = vu ? vu[k] : 0.0;
    coef[5 * k + 4] = phase[k];
  }
  if (psi) std::copy(psi, psi + (size_t)nth * ntc, ps.begin());
  if (wsevar) std::copy(wsevar, wsevar + nth, var.begin());
  if (f->ntc < ntc) {  // buffers for the largest constituent count set so far
    if (f->alloc(&f->d_tide, (size_t)ntc * 5) || f->alloc(&f->d_psi, (size_t)nth * ntc)) return CMS_DEVICE_ERROR;
  }
  if (!f->d_wsevar && f->alloc(&f->d_wsevar, (size_t)nth)) return CMS_DEVICE_ERROR;
  cudaStream_t s = f->S->stream;
  if (cudaMemcpyAsync(f->d_tide, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(f->d_psi, ps.data(), ps.size() * sizeof(double), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(f->d_wsevar, var.data(), var.size() * sizeof(double), cudaMemcpyHostToDevice, s) ||
      cudaStreamSynchronize(s))
    return CMS_DEVICE_ERROR;
  f->ntc = ntc;
  f->tide_dtj = dtj;
  f->tide_offset = offset;
  return CMS_OK;
}

int cms_flow_set_time(cms_flow* f, double t_seconds) {
  if (!f) return CMS_BAD_ARGUMENT;
  f->t_sim = t_seconds;
  return CMS_OK;
}

int cms_flow_get(cms_flow* f, int which, double* out) {
  if (!f || !out) return CMS_BAD_ARGUMENT;
  const int nD = f->nD, nmf = f->nmf;
  cms::FlowState& T = f->st;
  const double* cell = nullptr;
  const double* face = nullptr;
  if (which == CMS_FLOW_IWET) {  // the host copy is the one the device flags were made from
    for (int i = 0; i < nD; ++i) out[i] = f->geom.iwet[i];
    return CMS_OK;
  }
  switch (which) {
    case CMS_FLOW_P: cell = T.p; break;
    case CMS_FLOW_H: cell = T.h; break;
    case CMS_FLOW_U: cell = T.u; break;
    case CMS_FLOW_V: cell = T.v; break;
    case CMS_FLOW_ETA: cell = T.eta; break;
    case CMS_FLOW_VIS: cell = T.vis; break;
    case CMS_FLOW_CFRICT: cell = T.cfrict; break;
    case CMS_FLOW_DPX: cell = T.dpx[0]; break;
    case CMS_FLOW_DPY: cell = T.dpy[0]; break;
    case CMS_FLOW_FLUX: face = T.flux; break;
    case CMS_FLOW_VISK: face = T.visk; break;
    case CMS_FLOW_HK: face = T.hk; break;
    case CMS_FLOW_ACOEF: face = T.acoef; break;
    case CMS_FLOW_FINTP: face = f->G.fintp; break;
    case CMS_FLOW_ZBK: face = T.zbk; break;
    default: return CMS_BAD_ARGUMENT;
  }
  cudaStream_t s = f->S->stream;
  if (cell) {
    std::vector<double> h(nD);
    if (cudaMemcpyAsync(h.data(), cell, nD * sizeof(double), cudaMemcpyDeviceToHost, s) ||
        cudaStreamSynchronize(s))
      return CMS_DEVICE_ERROR;
    for (int r = 0; r < nD; ++r) out[f->d2n[r]] = h[r];
  } else {
    std::vector<double> h((size_t)nmf * nD);
    if (cudaMemcpyAsync(h.data(), face, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s) ||
        cudaStreamSynchronize(s))
      return CMS_DEVICE_ERROR;
    for (int r = 0; r < nD; ++r)
      for (int k = 0; k < nmf; ++k) out[(size_t)f->d2n[r] * nmf + k] = h[(size_t)k * nD + r];
  }
  return CMS_OK;
}

int cms_flow_last_info(const cms_flow* f, cms_flow_info* info) {
  if (!f || !info) return CMS_BAD_ARGUMENT;
  *info = f->last;
  return CMS_OK;
}

int cms_flow_last_solves(const cms_flow* f, cms_solve_info* info3) {
  if (!f || !info3) return CMS_BAD_ARGUMENT;
  for (int q = 0; q < 3; ++q) info3[q] = f->last_solve[q];
  return CMS_OK;
}

cms_solver* cms_flow_solver(cms_flow* f) { return f ? f->S : nullptr; }
long long cms_flow_launches(const cms_flow* f) { return f ? f->launches + (f->S ? f->S->launches : 0) : 0; }
size_t cms_flow_device_bytes(const cms_flow* f) { return f ? f->bytes + (f->S ? f->S->bytes : 0) : 0; }
int cms_flow_njoint(const cms_flow* f) { return f ? f->geom.njoint : -1; }

int cms_flow_wetdry_stats(const cms_flow* f, long long* updates, double* ms3) {
  if (!f || !updates || !ms3) return CMS_BAD_ARGUMENT;
  *updates = f->wd_updates;
  for (int q = 0; q < 3; ++q) ms3[q] = f->wd_ms[q];
  return CMS_OK;
}

int cms_flow_set_graphs(cms_flow* f, int on) {
  if (!f) return CMS_BAD_ARGUMENT;
  f->use_graphs = on ? 1 : 0;
  return CMS_OK;
}

int cms_flow_graph_stats(const cms_flow* f, long long* replays, long long* captures) {
  if (!f) return CMS_BAD_ARGUMENT;
  if (replays) *replays = f->graph_launches;
  if (captures) *captures = f->graph_captures;
  return CMS_OK;
}

void cms_flow_destroy(cms_flow* f) {
  if (!f) return;
  if (f->S) cudaStreamSynchronize(f->S->stream);
  for (auto& row : f->sgraph)
    for (auto& g : row)
      if (g.exec) cudaGraphExecDestroy(g.exec);
  for (void* p : f->allocs) cudaFree(p);
  if (f->h_flag) cudaFreeHost(f->h_flag);
  if (f->S) cms_solver_destroy(f->S);
  delete f;
}

}  // extern "C"
