// libcmsgpu: B200 (sm_100a) drop-in for CMS-Flow's solve() boundary.
//
// Host driver of the device kernels in cms_krylov.cuh.  One handle owns a CUDA
// stream, the device-order sparsity pattern and every work buffer; the
// per-call path allocates nothing once the handle has seen a call of the same
// precision.  Scalars of the Krylov recurrences stay on the device; the host
// only enqueues kernels and polls the device `done` flag between chunks of
// iterations, so a converged solve stops at exactly the iteration the
// reference's stopping test selects (later kernels see `done` and return).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cms_common.cuh"
#include "cms_krylov.cuh"
#include "cms_legacy.cuh"
#include "cms_order.h"
#include "cms_persist.cuh"
#include "cms_schur.cuh"
#include "cmsgpu.h"

static char g_last_error[512] = "";

namespace cms {

#define CMS_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      std::snprintf(g_last_error, sizeof(g_last_error), "%s:%d %s: %s", __FILE__, __LINE__, #call, \
                    cudaGetErrorString(e_));                                             \
      return CMS_DEVICE_ERROR;                                                           \
    }                                                                                    \
  } while (0)


template <typename T>
struct Mat {
  T* aoff = nullptr;
  T* diag = nullptr;
  T* luoff = nullptr;
  T* invd = nullptr;
};

template <typename T>
struct Work {
  T *b = nullptr, *x = nullptr, *r = nullptr, *r0 = nullptr, *p = nullptr, *u = nullptr, *v = nullptr, *z = nullptr;
  T* vv[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

template <typename T>
struct Staging {  // natural-order copies for the host-pointer entry points
  T *acoef = nullptr, *ss = nullptr, *sp = nullptr, *res = nullptr, *phi = nullptr;
};

}  // namespace cms

struct cms_solver {
  cms::HostPattern hp;
  cms_solver_opts opts{};
  cudaStream_t stream = nullptr;
  int dev = 0;
  // pattern
  int *d_perm = nullptr, *d_iperm = nullptr, *d_c2c = nullptr, *d_ncface = nullptr, *d_iwet = nullptr,
      *d_col = nullptr;
  signed char *d_fslot = nullptr, *d_nlo = nullptr, *d_nup = nullptr;
  int K = 0;
  cms::GroupTab tab{};           // all-row launches
  std::vector<int> gblocks; // blocks per group
  // numeric buffers
  cms::Mat<double> A64;
  cms::Mat<float> A32;
  cms::Mat<double> AT64;     // adjoint: A^T's values and its factor (diag shared with A64)
  int* d_tslot = nullptr;    // adjoint: transpose map of the ELL slots
  cms::Work<double> W64;
  cms::Work<float> W32;
  double* ir_r64 = nullptr;  // refinement: FP64 residual scratch (unused when null)
  cms::DevState* d_st = nullptr;
  cms::DevState* h_st = nullptr;  // pinned mirror
  double* d_part = nullptr;
  int max_blocks = 0;
  // persistent BiCGStab: slots per group, tile tables, block partials [2][3][tiles]
  int *d_gkl = nullptr, *d_gku = nullptr;
  int *d_toff = nullptr, *d_dep_ptr = nullptr, *d_dep_idx = nullptr;
  unsigned int* d_progress = nullptr;
  double* d_ppart = nullptr;
  int ptiles = 0;  // tiles (= blocks) of the persistent kernel; 0 not built, -1 not launchable
  size_t cap_toff = 0, cap_dep = 0;  // capacities of d_toff / d_dep_idx
  // reduced (Schur complement) inner solve of refinement (cms_schur.cuh):
  // Chat's pattern and values, 1/d and 1/s, neighbour tiles under Chat
  int sc_state = 0;  // 0 not built, 1 built, -1 not possible on this pattern
  int sc_KC = 0, sc_tiles = 0;
  int sc_sym = 0;    // Chat's pattern is structurally symmetric (d_sctr built)
  long long sc_nnz = 0, sc_e0b = 0;  // stored entries of Chat; couplings between group 0 and B
  int *d_sccol = nullptr, *d_sdep_ptr = nullptr, *d_sdep_idx = nullptr, *d_sctr = nullptr;
  float *d_scoff = nullptr, *d_ssinv = nullptr, *d_sst = nullptr;
  signed char* d_sccnt = nullptr;
  size_t cap_sdep = 0;
  long long reduced_fallbacks = 0;  // refinements finished on the exact factor after a bad inner correction
  int cur_relax = 0;  // the FP32 factor in A32 is the two-phase one (k_ilu0_relax)
  int cur_fuse = 0;   // inner solves of refinement: update folded into the next iteration
  // MATRIX_SOLVER options 1, 2, 5-8: compass table (built on first use),
  // its properties (-1 not built) and the 5-point solvers' scratch
  int* d_cmp = nullptr;
  int leg_props = -1;
  // pipelined passes (orderings with many groups): chunk table, per-row pass
  // counts, work-unit ticket, error flag, passes issued in the current solve
  int* d_pipe_cstart = nullptr;
  int pipe_nchunk = 0;
  unsigned int* d_pipe_done = nullptr;
  unsigned int* d_pipe_ticket = nullptr;
  int* d_pipe_err = nullptr;
  unsigned int pipe_epoch = 0;
  std::vector<int> pipe_gchunk;  // [G + 1] first chunk of each group
  int pipe_wave = 0;             // 1 + the largest group step to an upper neighbour
  int2* d_pipe_units = nullptr;  // wavefront order of the units of forward passes
  size_t pipe_units_cap = 0;
  int pipe_units_npass = 0;
  double* leg64 = nullptr;
  float* leg32 = nullptr;
  cms::Staging<double> S64;
  cms::Staging<float> S32;
  size_t bytes = 0;
  long long launches = 0;
  std::vector<void*> allocs;
  // optional per-kernel-class timing (CUDA events on the handle's stream)
  int prof_on = 0;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  struct ProfRec { int cat; size_t ev; double bytes; };
  std::vector<ProfRec> prof_recs;
  double prof_ms[16] = {0};  // per ProfCat
  double prof_bytes[16] = {0};
  long long prof_count[16] = {0};

  template <typename P>
  int alloc(P** p, size_t count) {
    size_t nb = std::max<size_t>(count, 1) * sizeof(P);
    CMS_CUDA(cudaMalloc((void**)p, nb));
    CMS_CUDA(cudaMemsetAsync(*p, 0, nb, stream));
    allocs.push_back((void*)*p);
    bytes += nb;
    return CMS_OK;
  }
};

namespace cms {

using Solver = ::cms_solver;

static inline int nblk(int rows) { return (rows + TPB - 1) / TPB; }
// Grid of a row kernel: one row per thread up to 8 blocks of 256 threads per
// SM on the 148 SMs, grid-stride beyond that (fewer block partials to reduce,
// more rows in flight per thread).
constexpr int GRID_CAP = 148 * 8;
static inline int gsz(int rows) { return std::max(1, std::min(nblk(rows), GRID_CAP)); }

#define CHK(...)                     \
  do {                               \
    int rc_ = (__VA_ARGS__);         \
    if (rc_ != CMS_OK) return rc_;   \
  } while (0)

#define LAUNCH_CHECK(S)                          \
  do {                                           \
    (S)->launches++;                             \
    cudaError_t e_ = cudaGetLastError();         \
    if (e_ != cudaSuccess) {                     \
      std::snprintf(g_last_error, sizeof(g_last_error), "launch: %s", cudaGetErrorString(e_)); \
      return CMS_DEVICE_ERROR;                   \
    }                                            \
  } while (0)

// Kernel classes timed by the profiler (cms_solver_profile_*).
enum ProfCat : int {
  P_PROLOGUE = 0, P_ILU0 = 1, P_FWD = 2, P_BWD = 3, P_SPMV = 4, P_VEC = 5, P_RESID64 = 6, P_SCALAR = 7,
  P_FLOW = 8, P_PERSIST = 9, P_SCHUR_BUILD = 10, P_SCHUR = 11, P_NCAT = 12
};

static void prof_begin(Solver* S) {
  if (!S->prof_on) return;
  if (S->ev_used + 2 > S->ev_pool.size()) {
    for (int q = 0; q < 256; ++q) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) { S->prof_on = 0; return; }
      S->ev_pool.push_back(e);
    }
  }
  cudaEventRecord(S->ev_pool[S->ev_used], S->stream);
}

static void prof_end(Solver* S, int cat, double bytes) {
  if (!S->prof_on) return;
  cudaEventRecord(S->ev_pool[S->ev_used + 1], S->stream);
  S->prof_recs.push_back({cat, S->ev_used, bytes});
  S->ev_used += 2;
}

// Launch with error check, launch count and optional timing; BYTES are the
// algorithmic bytes of the launch (each array the kernel touches counted once).
#define KLAUNCH(S, CAT, BYTES, ...)   \
  do {                                \
    prof_begin(S);                    \
    __VA_ARGS__;                      \
    LAUNCH_CHECK(S);                  \
    prof_end(S, CAT, (double)(BYTES)); \
  } while (0)

template <typename T>
static int alloc_precision(Solver* S, Mat<T>& A, Work<T>& W) {
  const size_t n = S->hp.n, K = std::max(S->K, 1);
  CHK(S->alloc(&A.aoff, K * n));
  CHK(S->alloc(&A.diag, n));
  CHK(S->alloc(&A.luoff, K * n));
  CHK(S->alloc(&A.invd, n));
  CHK(S->alloc(&W.b, n));
  CHK(S->alloc(&W.x, n));
  CHK(S->alloc(&W.r, n));
  CHK(S->alloc(&W.r0, n));
  CHK(S->alloc(&W.p, n));
  CHK(S->alloc(&W.u, n));
  CHK(S->alloc(&W.v, n));
  CHK(S->alloc(&W.z, n));
  for (int j = 1; j <= 4; ++j) CHK(S->alloc(&W.vv[j], n));
  return CMS_OK;
}

template <typename T>
static int alloc_staging(Solver* S, Staging<T>& st) {
  if (st.acoef) return CMS_OK;
  const size_t nD = S->hp.nD, nmf = S->hp.nmf;
  CHK(S->alloc(&st.acoef, nD * nmf));
  CHK(S->alloc(&st.ss, nD));
  CHK(S->alloc(&st.sp, nD));
  CHK(S->alloc(&st.res, nD));
  CHK(S->alloc(&st.phi, nD));
  return CMS_OK;
}

static int create(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface, const int* iwet,
                  const cms_solver_opts* opts, Solver** out) {
  if (!out || !cell2cell || !ncface || ncells <= 0 || ncellsD < ncells || nmaxfaces <= 0 || nmaxfaces > KMAX)
    return CMS_BAD_ARGUMENT;
  auto* S = new cms_solver();
  if (opts) S->opts = *opts; else cms_solver_default_opts(&S->opts);
  std::string err = build_pattern(ncells, ncellsD, nmaxfaces, cell2cell, ncface, S->opts.ordering, S->hp);
  if (!err.empty()) {
    std::snprintf(g_last_error, sizeof(g_last_error), "%s", err.c_str());
    delete S;
    return CMS_BAD_ARGUMENT;
  }
  HostPattern& P = S->hp;
  if (P.KL > KMAX || P.KU > KMAX) {
    std::snprintf(g_last_error, sizeof(g_last_error), "more than %d lower/upper couplings in a row", KMAX);
    delete S;
    return CMS_UNSUPPORTED;
  }
  S->K = P.KL + P.KU;
  int rc = CMS_OK;
  auto fail = [&](int code) { cms_solver_destroy(S); return code; };
  if (cudaGetDevice(&S->dev) != cudaSuccess) return fail(CMS_DEVICE_ERROR);
  if (cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(CMS_DEVICE_ERROR);
  const size_t n = P.n, nD = P.nD, nmf = P.nmf, K = std::max(S->K, 1);
  if ((rc = S->alloc(&S->d_perm, n)) || (rc = S->alloc(&S->d_iperm, n)) || (rc = S->alloc(&S->d_c2c, nD * nmf)) ||
      (rc = S->alloc(&S->d_ncface, nD)) || (rc = S->alloc(&S->d_iwet, nD)) || (rc = S->alloc(&S->d_col, K * n)) ||
      (rc = S->alloc(&S->d_fslot, n * nmf)) || (rc = S->alloc(&S->d_nlo, n)) || (rc = S->alloc(&S->d_nup, n)))
    return fail(rc);
  cudaStream_t s = S->stream;
  if (cudaMemcpyAsync(S->d_perm, P.perm.data(), n * sizeof(int), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(S->d_iperm, P.iperm.data(), n * sizeof(int), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(S->d_c2c, cell2cell, nD * nmf * sizeof(int), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(S->d_ncface, ncface, nD * sizeof(int), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(S->d_col, P.col.data(), P.col.size() * sizeof(int), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(S->d_fslot, P.fslot.data(), n * nmf, cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(S->d_nlo, P.nlo.data(), n, cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(S->d_nup, P.nup.data(), n, cudaMemcpyHostToDevice, s))
    return fail(CMS_DEVICE_ERROR);
  {
    std::vector<int> w(nD, 1);
    if (iwet) std::memcpy(w.data(), iwet, nD * sizeof(int));
    if (cudaMemcpyAsync(S->d_iwet, w.data(), nD * sizeof(int), cudaMemcpyHostToDevice, s) ||
        cudaStreamSynchronize(s))
      return fail(CMS_DEVICE_ERROR);
  }
  // group tables
  S->gblocks.resize(P.G);
  int tot = 0;
  for (int g = 0; g < P.G; ++g) {
    const int rows = P.gstart[g + 1] - P.gstart[g];
    const long long prop = ((long long)GRID_CAP * rows + P.n - 1) / P.n;
    S->gblocks[g] = std::max(1, (int)std::min<long long>(nblk(rows), std::max<long long>(prop, 1)));
    tot += S->gblocks[g];
  }
  GroupTab& t = S->tab;
  std::memset(&t, 0, sizeof(t));
  if (P.G <= MAXG) {
    t.ng = P.G;
    int b = 0;
    for (int g = 0; g < P.G; ++g) {
      t.start[g] = P.gstart[g];
      t.blk[g] = b;
      t.kl[g] = P.gkl[g];
      t.ku[g] = P.gku[g];
      b += S->gblocks[g];
    }
    t.start[P.G] = P.gstart[P.G];
    t.blk[P.G] = b;
  } else {  // level schedule: one merged group with the global slot bounds
    t.ng = 1;
    t.start[0] = 0;
    t.start[1] = P.n;
    t.blk[0] = 0;
    t.blk[1] = gsz(P.n);
    t.kl[0] = P.KL;
    t.ku[0] = P.KU;
  }
  // every reduction kernel launches at most max(GRID_CAP, table blocks) blocks
  S->max_blocks = std::max(std::max(tot, GRID_CAP), std::max(t.blk[t.ng], gsz(P.n))) + 1;
  if ((rc = S->alloc(&S->d_part, (size_t)3 * S->max_blocks)) || (rc = S->alloc(&S->d_st, 1))) return fail(rc);
  if ((rc = S->alloc(&S->d_gkl, P.G)) || (rc = S->alloc(&S->d_gku, P.G)) ||
      (rc = S->alloc(&S->d_ppart, (size_t)2 * NSMAX * GRID_CAP)))
    return fail(rc);
  if (cudaMemcpyAsync(S->d_gkl, P.gkl.data(), P.G * sizeof(int), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(S->d_gku, P.gku.data(), P.G * sizeof(int), cudaMemcpyHostToDevice, s))
    return fail(CMS_DEVICE_ERROR);
  if (cudaMallocHost((void**)&S->h_st, sizeof(DevState)) != cudaSuccess) return fail(CMS_DEVICE_ERROR);
  if ((rc = alloc_precision(S, S->A64, S->W64)) || (rc = alloc_precision(S, S->A32, S->W32))) return fail(rc);
  if (cudaStreamSynchronize(s) != cudaSuccess) return fail(CMS_DEVICE_ERROR);
  *out = S;
  return CMS_OK;
}

// ---------------------------------------------------------------------------
// Launch helpers

template <typename T>
static int factor(Solver* S, Mat<T>& A) {
  const HostPattern& P = S->hp;
  const double s = sizeof(T);
  for (int g = 0; g < P.G; ++g) {
    const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
    if (r1 <= r0) continue;
    const double R = r1 - r0, E = (double)(P.glo[g] + P.gup[g]);
    KLAUNCH(S, P_ILU0, R * (3 * s + 1) + E * (2 * s + 4),
            (k_ilu0<T><<<gsz(r1 - r0), TPB, 0, S->stream>>>(P.n, r0, r1, P.KL, P.gkl[g], P.gku[g], S->d_col,
                                                             S->d_nlo, S->d_nup, A.aoff, A.diag, A.luoff, A.invd)));
  }
  return CMS_OK;
}

template <typename T, int MODE>
static int sweep_fwd(Solver* S, Mat<T>& A, Work<T>& W, int step, const T* yin, T* p, T* r, const T* u, T* x) {
  const HostPattern& P = S->hp;
  const double s = sizeof(T);
  // vectors streamed per row by each mode (reads + writes)
  const double vec = MODE == FWD_PLAIN ? 2 : MODE == FWD_BICG_P ? 5 : MODE == FWD_BICG_R ? 7 : MODE == FWD_GM_SCALE ? 3 : 4;
  GmVecs gv;
  for (int j = 0; j < 5; ++j) gv.v[j] = W.vv[j];
  for (int g = 0; g < P.G; ++g) {
    const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
    if (r1 <= r0) continue;
    const double R = r1 - r0, E = (double)P.glo[g];
    KLAUNCH(S, P_FWD, R * s * vec + E * (s + 4) + (E > 0 ? R * s : 0.0),
            (k_fwd<T, MODE><<<gsz(r1 - r0), TPB, 0, S->stream>>>(P.n, r0, r1, P.gkl[g], step, S->d_col, S->d_nlo,
                                                                  A.luoff, W.z, yin, p, r, u, x, gv, S->d_st)));
  }
  return CMS_OK;
}

template <typename T, bool FINAL>
static int sweep_bwd(Solver* S, Mat<T>& A, Work<T>& W, T* x, int need_active) {
  const HostPattern& P = S->hp;
  const double s = sizeof(T);
  for (int g = P.G - 1; g >= 0; --g) {
    const int r0 = P.gstart[g], r1 = P.gstart[g + 1];
    if (r1 <= r0) continue;
    const double R = r1 - r0, E = (double)P.gup[g];
    KLAUNCH(S, P_BWD, R * s * (FINAL ? 5 : 3) + E * (s + 4) + (E > 0 ? R * s : 0.0),
            (k_bwd<T, FINAL><<<gsz(r1 - r0), TPB, 0, S->stream>>>(P.n, r0, r1, P.KL, P.gku[g], S->d_col, S->d_nup,
                                                                   A.luoff, A.invd, W.z, x, need_active, S->d_st)));
  }
  return CMS_OK;
}

static int poll_done(Solver* S, bool& done) {
  CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  done = S->h_st->done != 0;
  return CMS_OK;
}

// algorithmic bytes of one all-row matrix pass: diag + ELL values/indices + nvec vectors
template <typename T>
static double spmv_bytes(const Solver* S, double nvec) {
  return (double)S->hp.n * sizeof(T) * (1 + nvec) + (double)S->hp.nnz_off * (sizeof(T) + 4);
}

// One BiCGStab iteration (pbicgstab.f90:41-96) = 4G + 3 launches.
template <typename T>
static int bicg_iter(Solver* S, Mat<T>& A, Work<T>& W) {
  const HostPattern& P = S->hp;
  const int nb_all = S->tab.blk[S->tab.ng];
  CHK((sweep_fwd<T, FWD_BICG_P>(S, A, W, 0, nullptr, W.p, W.r, W.u, W.x)));
  CHK((sweep_bwd<T, false>(S, A, W, nullptr, 0)));
  KLAUNCH(S, P_SPMV, spmv_bytes<T>(S, 3),
          (k_spmv<T, SPMV_BICG_U><<<nb_all, TPB, 0, S->stream>>>(P.n, P.KL, S->tab, 0, S->d_col, S->d_nlo, S->d_nup,
                                                                  A.aoff, A.diag, W.z, W.u, W.r0, S->d_part,
                                                                  S->d_st)));
  CHK((sweep_fwd<T, FWD_BICG_R>(S, A, W, 0, nullptr, W.p, W.r, W.u, W.x)));
  CHK((sweep_bwd<T, false>(S, A, W, nullptr, 0)));
  KLAUNCH(S, P_SPMV, spmv_bytes<T>(S, 3),
          (k_spmv<T, SPMV_BICG_V><<<nb_all, TPB, 0, S->stream>>>(P.n, P.KL, S->tab, 0, S->d_col, S->d_nlo, S->d_nup,
                                                                  A.aoff, A.diag, W.z, W.v, W.r, S->d_part,
                                                                  S->d_st)));
  KLAUNCH(S, P_VEC, (double)P.n * sizeof(T) * 7,
          (k_bicg_update<T><<<gsz(P.n), TPB, 0, S->stream>>>(P.n, W.z, W.v, W.x, W.r, W.r0, S->d_part, S->d_st)));
  return CMS_OK;
}

// Blocks of the persistent kernels that can be resident at once on the
// device (cooperative launch limit); 0 when it cannot be launched.
static int persist_capacity(int dev) {
  int coop = 0, nsm = 0, per32 = 0, per64 = 0, perb = 0, pers = 0, persb = 0, persr = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per32, k_bicg_persistent<float>, TPB, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per64, k_bicg_persistent<double>, TPB, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perb, k_bicg_batched<float>, TPB, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pers, k_schur_bicg<TPB, 2, 0>, TPB, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&persb, k_schur_batched<TPB, 2, 0>, TPB, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&persr, k_schur_batched<TPB, 2, 1>, TPB, 0) != cudaSuccess ||
      std::min(std::min(std::min(std::min(std::min(per32, per64), perb), pers), persb), persr) <= 0) {
    cudaGetLastError();
    return 0;
  }
  return std::min(std::min(std::min(std::min(std::min(std::min(per32, per64), perb), pers), persb), persr) * nsm,
                  GRID_CAP);
}

static int build_tiles(Solver* S, int nt);

// Tiles of the persistent kernel: one block per tile, every block resident,
// at most one block per 256 rows.  Builds the tile tables on first use; 0
// when the device cannot launch the kernel or a group does not keep natural
// order.
static int persist_tiles(Solver* S) {
  if (S->ptiles != 0) return std::max(S->ptiles, 0);
  const int cap = persist_capacity(S->dev);
  if (cap <= 0) {
    S->ptiles = -1;
    return 0;
  }
  return build_tiles(S, std::min(cap, nblk(S->hp.n)));
}

// Tile tables for nt tiles (tile t = natural cells [t n / nt, (t+1) n / nt)).
static int build_tiles(Solver* S, int nt) {
  const HostPattern& P = S->hp;
  const int n = P.n;
  nt = std::max(1, std::min(std::min(nt, nblk(n)), GRID_CAP));
  if (S->ptiles == nt) return nt;
  S->ptiles = -1;
  // tile t = natural cells [tstart[t], tstart[t+1])
  std::vector<int> tstart(nt + 1), tile_nat(n);
  for (int t = 0; t <= nt; ++t) tstart[t] = (int)((long long)t * n / nt);
  for (int t = 0; t < nt; ++t)
    for (int i = tstart[t]; i < tstart[t + 1]; ++i) tile_nat[i] = t;
  std::vector<int> toff((size_t)P.G * (nt + 1));
  for (int g = 0; g < P.G; ++g) {
    int r = P.gstart[g];
    for (int q = r + 1; q < P.gstart[g + 1]; ++q)
      if (P.perm[q] <= P.perm[q - 1]) return 0;  // rows of a group must keep natural order
    for (int t = 0; t <= nt; ++t) {
      while (r < P.gstart[g + 1] && P.perm[r] < tstart[t]) ++r;
      toff[(size_t)g * (nt + 1) + t] = r;
    }
  }
  // neighbour tiles (symmetric): tiles holding a row coupled to one of ours
  std::vector<std::vector<int>> dep(nt);
  auto add = [&](int a, int b) {
    for (int q : dep[a]) if (q == b) return;
    dep[a].push_back(b);
  };
  for (int r = 0; r < n; ++r) {
    const int ti = tile_nat[P.perm[r]];
    for (int s = 0; s < S->K; ++s) {
      const int j = P.col[(size_t)s * n + r];
      if (j == r) continue;
      const int tj = tile_nat[P.perm[j]];
      if (tj != ti) { add(ti, tj); add(tj, ti); }
    }
  }
  std::vector<int> dptr(nt + 1, 0), didx;
  for (int t = 0; t < nt; ++t) {
    std::sort(dep[t].begin(), dep[t].end());
    didx.insert(didx.end(), dep[t].begin(), dep[t].end());
    dptr[t + 1] = (int)didx.size();
  }
  // buffers sized for the largest table built so far
  if (toff.size() > S->cap_toff) {
    if (S->alloc(&S->d_toff, toff.size())) return 0;
    S->cap_toff = toff.size();
  }
  if (didx.size() + 1 > S->cap_dep) {
    if (S->alloc(&S->d_dep_idx, didx.size() + 1)) return 0;
    S->cap_dep = didx.size() + 1;
  }
  if (!S->d_dep_ptr && (S->alloc(&S->d_dep_ptr, GRID_CAP + 1) || S->alloc(&S->d_progress, (size_t)GRID_CAP * kProgressStride))) return 0;
  cudaStream_t s = S->stream;
  if (cudaMemcpyAsync(S->d_toff, toff.data(), toff.size() * sizeof(int), cudaMemcpyHostToDevice, s) ||
      cudaMemcpyAsync(S->d_dep_ptr, dptr.data(), dptr.size() * sizeof(int), cudaMemcpyHostToDevice, s) ||
      (!didx.empty() &&
       cudaMemcpyAsync(S->d_dep_idx, didx.data(), didx.size() * sizeof(int), cudaMemcpyHostToDevice, s)) ||
      cudaStreamSynchronize(s))
    return 0;
  S->ptiles = nt;
  return nt;
}

// Algorithmic bytes of one persistent launch (each array a phase touches
// counted once per phase): the start, then per iteration two preconditioner
// applications (forward phases with their right-hand side formed in place,
// backward phases), two SpMVs with their dot products and the x/r update.
// The last forward group does its backward step in place (relax: every group
// after the first); with spmv0 the backward phase of group 0 also forms the
// SpMV of its rows from the same column indices and gathered values.
template <typename T>
static double persist_bytes(const Solver* S, int iters, bool xzero, bool relax, bool spmv0) {
  const HostPattern& P = S->hp;
  const double s = sizeof(T), n = P.n;
  const bool fuse = relax || (P.G > 0 && P.gku[P.G - 1] == 0);
  double fwd = 0.0, bwd = 0.0, spmv_rest = 0.0;
  for (int g = 0; g < P.G; ++g) {
    const double R = P.gstart[g + 1] - P.gstart[g], El = P.glo[g], Eu = P.gup[g];
    fwd += El * (s + 4) + (El > 0 ? R * s : 0.0);  // factor entries, columns, gathered values
    const bool last = fuse && (g == P.G - 1 || (relax && g >= 1));
    if (last) fwd += R * s;                         // invd
    if (g == 0 && spmv0) {
      // backward step of group 0 fused with its SpMV rows: z, diag, dot
      // operand in; z, output out; A's entries (the factor's rows of group 0
      // are A's), columns, gathered values
      bwd += R * s * 5 + Eu * (s + 4) + (Eu > 0 ? R * s : 0.0);
      continue;
    }
    if (!last) bwd += R * s * 3 + Eu * (s + 4) + (Eu > 0 ? R * s : 0.0);
    // SpMV: diag, own value, output, dot operand, matrix entries, columns, gathers
    spmv_rest += R * s * 4 + (El + Eu) * (s + 4) + (El + Eu > 0 ? R * s : 0.0);
  }
  // forward right-hand sides: p-update reads r, p, u, writes p, z (5); x/r
  // update reads z, x, r, u, writes x, r, z (7)
  const double it = 2 * (fwd + bwd + spmv_rest) + n * s * (5 + 7) + n * s * 7;
  const double start = xzero ? n * s * 7 : spmv_bytes<T>(S, 7);
  return start + iters * it;
}

// Arguments of the persistent kernel for one system (tile count set by the
// caller: gridDim for one system, the member's tiles in a batch).
template <typename T>
static PersistArgs<T> make_args(Solver* S, Mat<T>& A, Work<T>& W, int tiles, int maxit, int norm, double tol,
                                int xzero) {
  const HostPattern& P = S->hp;
  PersistArgs<T> a;
  std::memset(&a, 0, sizeof(a));
  a.n = P.n; a.KL = P.KL; a.KU = P.KU; a.G = P.G; a.gku_last = P.gku[P.G - 1];
  a.klB = a.kuB = 0;
  for (int g = 1; g < P.G; ++g) {
    a.klB = std::max(a.klB, P.gkl[g]);
    a.kuB = std::max(a.kuB, P.gku[g]);
  }
  a.ntiles = tiles;
  a.gkl = S->d_gkl; a.gku = S->d_gku;
  a.toff = S->d_toff; a.dep_ptr = S->d_dep_ptr; a.dep_idx = S->d_dep_idx; a.progress = S->d_progress;
  a.col = S->d_col; a.nlo = S->d_nlo; a.nup = S->d_nup;
  a.aoff = A.aoff; a.diag = A.diag; a.luoff = A.luoff; a.invd = A.invd;
  a.b = W.b; a.x = W.x; a.r = W.r; a.r0 = W.r0; a.p = W.p; a.u = W.u; a.v = W.v; a.z = W.z;
  a.part = S->d_ppart; a.bar = &S->d_st->bar; a.st = S->d_st;
  a.maxit = maxit; a.norm = norm; a.xzero = xzero; a.tol = tol;
  a.spin_limit = kSpinLimit;
  a.relax = S->cur_relax;
  a.fuse_upd = (S->cur_fuse && norm == 2) ? 1 : 0;
  a.g1 = P.G > 1 ? P.gstart[1] : P.n;
  a.spmv0 = (P.gkl[0] == 0 && ((a.relax || a.gku_last == 0) ? P.G >= 2 : P.G >= 1)) ? 1 : 0;
  return a;
}

// Runs one of the persistent kernel's waits (which = 0 neighbour wait, 1
// grid barrier) on a two-tile table whose second tile never runs, with a
// limit of spin_limit polls, on scratch of its own (the handle's tables are
// untouched).  CMS_DEVICE_ERROR with the message is the expected result.
static int persist_wait_selftest(Solver* S, unsigned int spin_limit, int which) {
  // one buffer: progress [2 * stride], dep_ptr [3], dep_idx [2], GridBar, out [2]
  const size_t nprog = 2 * kProgressStride;
  const size_t words = nprog + 3 + 2 + sizeof(GridBar) / sizeof(unsigned int) + 2;
  unsigned int* buf = nullptr;
  CMS_CUDA(cudaMalloc((void**)&buf, words * sizeof(unsigned int)));
  struct Free { unsigned int* p; ~Free() { cudaFree(p); } } fr{buf};
  int* dep_ptr = reinterpret_cast<int*>(buf + nprog);
  int* dep_idx = dep_ptr + 3;
  GridBar* bar = reinterpret_cast<GridBar*>(dep_idx + 2);
  int* out = reinterpret_cast<int*>(bar + 1);
  const int h_dep[5] = {0, 1, 2, 1, 0};  // tile 0 depends on tile 1 and tile 1 on tile 0
  CMS_CUDA(cudaMemsetAsync(buf, 0, words * sizeof(unsigned int), S->stream));
  CMS_CUDA(cudaMemcpyAsync(dep_ptr, h_dep, sizeof(h_dep), cudaMemcpyHostToDevice, S->stream));
  PersistArgs<float> a;
  std::memset(&a, 0, sizeof(a));
  a.dep_ptr = dep_ptr; a.dep_idx = dep_idx; a.progress = buf; a.bar = bar; a.st = S->d_st;
  a.spin_limit = spin_limit;
  k_persist_wait_probe<float><<<1, TPB, 0, S->stream>>>(a, which, out);
  CMS_CUDA(cudaGetLastError());
  S->launches++;
  int h_out[2] = {0, 0};
  GridBar h_bar{};
  CMS_CUDA(cudaMemcpyAsync(h_out, out, sizeof(h_out), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaMemcpyAsync(&h_bar, bar, sizeof(GridBar), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  if (h_out[0] == 1 && h_bar.err == 1) {
    if (which == 0)
      std::snprintf(g_last_error, sizeof(g_last_error),
                    "persistent kernel: the neighbour wait gave up after %u polls (tile 1 never completed phase 1)",
                    spin_limit);
    else
      std::snprintf(g_last_error, sizeof(g_last_error),
                    "persistent kernel: the grid barrier gave up after %u polls (%d of 2 blocks arrived)", spin_limit,
                    h_out[1]);
    return CMS_DEVICE_ERROR;
  }
  std::snprintf(g_last_error, sizeof(g_last_error), "persistent kernel wait self-test: the wait did not give up");
  return CMS_OK;
}

// The whole BiCGStab solve as one cooperative launch.  Returns 1 (nothing
// enqueued but a memset) when the launch was refused for its size, so the
// caller can fall back to the per-phase kernels.
template <typename T>
static int run_bicgstab_persistent(Solver* S, Mat<T>& A, Work<T>& W, int tiles, int maxit, int norm, double tol,
                                   int xzero) {
  PersistArgs<T> a = make_args<T>(S, A, W, tiles, maxit, norm, tol, xzero);
  CMS_CUDA(cudaMemsetAsync(&S->d_st->bar, 0, sizeof(GridBar), S->stream));
  CMS_CUDA(cudaMemsetAsync(S->d_progress, 0, sizeof(unsigned int) * tiles * kProgressStride, S->stream));
  void* args[] = {&a};
  prof_begin(S);
  const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_bicg_persistent<T>, dim3(tiles), dim3(TPB), args,
                                                    0, S->stream);
  if (e == cudaErrorCooperativeLaunchTooLarge) {
    cudaGetLastError();
    S->ptiles = -1;
    return 1;
  }
  if (e != cudaSuccess) {
    std::snprintf(g_last_error, sizeof(g_last_error), "cooperative launch: %s", cudaGetErrorString(e));
    return CMS_DEVICE_ERROR;
  }
  S->launches++;
  const size_t nrec = S->prof_recs.size();
  prof_end(S, P_PERSIST, 0.0);
  const bool recorded = S->prof_recs.size() > nrec;
  CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  if (S->h_st->bar.err) {
    std::snprintf(g_last_error, sizeof(g_last_error), "persistent BiCGStab: a grid barrier wait timed out");
    return CMS_DEVICE_ERROR;
  }
  if (recorded) S->prof_recs.back().bytes = persist_bytes<T>(S, S->h_st->iter, xzero != 0, a.relax != 0, a.spmv0 != 0);
  return CMS_OK;
}

// BiCGStab from x (or 0) on b, ending when the device stopping test fires.
template <typename T>
static int run_bicgstab(Solver* S, Mat<T>& A, Work<T>& W, int maxit, int norm, double tol, int xzero,
                        bool do_factor = true) {
  const HostPattern& P = S->hp;
  const int nb_all = S->tab.blk[S->tab.ng];
  if (do_factor) CHK(factor<T>(S, A));
  if (!S->opts.multi_kernel) {
    const int tiles = persist_tiles(S);
    if (tiles > 0) {
      const int rc = run_bicgstab_persistent<T>(S, A, W, tiles, maxit, norm, tol, xzero);
      if (rc != 1) return rc;
    }
  }
  if (S->cur_relax) {  // the per-phase kernels need the exact factor
    S->cur_relax = 0;
    CHK(factor<T>(S, A));
  }
  KLAUNCH(S, P_VEC, xzero ? (double)P.n * sizeof(T) * 7 : spmv_bytes<T>(S, 7),
          (k_bicg_init<T><<<nb_all, TPB, 0, S->stream>>>(P.n, P.KL, S->tab, xzero, maxit, norm, tol, S->d_col,
                                                          S->d_nlo, S->d_nup, A.aoff, A.diag, W.b, W.x, W.r, W.r0,
                                                          W.p, W.u, W.v, S->d_part, S->d_st)));
  int issued = 0, chunk = S->prof_on ? 1 : 2;
  while (issued < maxit) {
    const int c = std::min(chunk, maxit - issued);
    for (int q = 0; q < c; ++q) CHK(bicg_iter<T>(S, A, W));
    issued += c;
    bool done = false;
    CHK(poll_done(S, done));
    if (done) break;
    if (!S->prof_on) chunk = std::min(chunk * 2, 16);
  }
  return CMS_OK;
}

// GMRES(3) restarts (pgmres.f90:129-241).
template <typename T>
static int run_gmres(Solver* S, Mat<T>& A, Work<T>& W, int maxit, double tol, bool do_factor = true) {
  const HostPattern& P = S->hp;
  const int nb_all = S->tab.blk[S->tab.ng];
  const double vb = (double)P.n * sizeof(T);
  if (do_factor) CHK(factor<T>(S, A));
  KLAUNCH(S, P_SCALAR, 0, (k_gm_start<<<1, 1, 0, S->stream>>>(S->d_st, maxit, tol)));
  GmVecs gv;
  for (int j = 0; j < 5; ++j) gv.v[j] = W.vv[j];
  for (int cyc = 0; cyc < maxit; ++cyc) {
    KLAUNCH(S, P_VEC, spmv_bytes<T>(S, 3),
            (k_gm_resid<T><<<nb_all, TPB, 0, S->stream>>>(P.n, P.KL, S->tab, S->d_col, S->d_nlo, S->d_nup, A.aoff,
                                                           A.diag, W.b, W.x, W.vv[1], S->d_part, S->d_st)));
    for (int i = 1; i <= 3; ++i) {
      CHK((sweep_fwd<T, FWD_GM_SCALE>(S, A, W, i, nullptr, nullptr, nullptr, nullptr, nullptr)));
      CHK((sweep_bwd<T, false>(S, A, W, nullptr, 1)));
      KLAUNCH(S, P_SPMV, spmv_bytes<T>(S, 3),
              (k_spmv<T, SPMV_GM><<<nb_all, TPB, 0, S->stream>>>(P.n, P.KL, S->tab, i, S->d_col, S->d_nlo, S->d_nup,
                                                                  A.aoff, A.diag, W.z, W.vv[i + 1], W.vv[1],
                                                                  S->d_part, S->d_st)));
      for (int j = 1; j <= i; ++j) {
        KLAUNCH(S, P_VEC, vb * 4, (k_mgs<T><<<gsz(P.n), TPB, 0, S->stream>>>(P.n, j, i, gv, S->d_part, S->d_st)));
      }
    }
    CHK((sweep_fwd<T, FWD_GM_COMB>(S, A, W, 0, nullptr, nullptr, nullptr, nullptr, nullptr)));
    CHK((sweep_bwd<T, true>(S, A, W, W.x, 0)));
    KLAUNCH(S, P_SCALAR, 0, (k_gm_cycle_end<<<1, 1, 0, S->stream>>>(S->d_st)));
    if (S->prof_on || (cyc & 1) || cyc + 1 == maxit) {
      bool done = false;
      CHK(poll_done(S, done));
      if (done) break;
    }
  }
  return CMS_OK;
}

template <typename T>
static int run_krylov(Solver* S, Mat<T>& A, Work<T>& W, int nsolv, int maxit, int norm, double tol, int xzero) {
  if (nsolv == 3) return run_bicgstab<T>(S, A, W, maxit, norm, tol, xzero);
  if (nsolv == 4) {
    if (xzero) {
      CMS_CUDA(cudaMemsetAsync(W.x, 0, sizeof(T) * S->hp.n, S->stream));
    }
    return run_gmres<T>(S, A, W, maxit, tol);
  }
  return CMS_UNSUPPORTED;
}

}  // namespace cms
#include "cms_legacy_host.cuh"
namespace cms {

// FP64 residual norm^2 of the device-order system into slot (A in TA, x in TX).
template <typename TA, typename TX>
static int resid64(Solver* S, Mat<TA>& A, const double* b, const TX* x, double* rout, float* rout32, int slot) {
  const HostPattern& P = S->hp;
  const double bytes = (double)P.n * (sizeof(TA) + 8 + sizeof(TX) + (rout ? 8 : 0) + (rout32 ? 4 : 0)) +
                       (double)P.nnz_off * (sizeof(TA) + 4);
  KLAUNCH(S, P_RESID64, bytes,
          (k_resid64<TA, TX><<<S->tab.blk[S->tab.ng], TPB, 0, S->stream>>>(P.n, P.KL, S->tab, S->d_col, S->d_nlo,
                                                                            S->d_nup, A.aoff, A.diag, b, x, rout,
                                                                            rout32, slot, S->d_part, S->d_st)));
  return CMS_OK;
}

// Pattern of the reduced inner system (cms_schur.cuh): Chat's columns per B
// row (direct couplings to B rows and the B neighbours of each group-0
// neighbour, the row itself excluded), once per handle; the neighbour-tile
// lists under Chat for the persistent tiles, rebuilt when the tile count
// changes.  CMS_UNSUPPORTED when the ordering has no independent first group
// or a reduced row has more than KSC entries.
static int schur_pattern(Solver* S, int tiles) {
  const HostPattern& P = S->hp;
  const int n = P.n;
  if (S->sc_state < 0) return CMS_UNSUPPORTED;
  if (S->sc_state == 0) {
    S->sc_state = -1;
    if (P.G < 2 || P.G > GFLAT || P.gkl[0] != 0) return CMS_UNSUPPORTED;
    const int g1 = P.gstart[1], nB = n - g1;
    if (g1 <= 0 || nB <= 0) return CMS_UNSUPPORTED;
    std::vector<int> tmp((size_t)nB * KSC);
    std::vector<signed char> cnt(nB);
    int KC = 0;
    long long nnz = 0, e0b = 0;
    for (int j = 0; j < g1; ++j) e0b += P.nup[j];
    for (int i = 0; i < nB; ++i) {
      const int r = g1 + i;
      int loc[8 * KMAX];
      int m = 0;
      const int kl = P.nlo[r], ku = P.nup[r];
      for (int s = 0; s < kl + ku; ++s) {
        const int k = P.col[(size_t)(s < kl ? s : P.KL + (s - kl)) * n + r];
        if (k >= g1) {
          loc[m++] = k;
          continue;
        }
        for (int t = 0; t < P.nup[k]; ++t) {
          const int k2 = P.col[(size_t)(P.KL + t) * n + k];
          if (k2 != r && m < 8 * KMAX) loc[m++] = k2;
        }
      }
      std::sort(loc, loc + m);
      const int mc = (int)(std::unique(loc, loc + m) - loc);
      if (mc > KSC) return CMS_UNSUPPORTED;
      std::copy(loc, loc + mc, tmp.begin() + (size_t)i * KSC);
      cnt[i] = (signed char)mc;
      KC = std::max(KC, mc);
      nnz += mc;
    }
    KC = std::max(KC, 1);
    std::vector<int> ccol((size_t)KC * nB);
    for (int i = 0; i < nB; ++i)
      for (int q = 0; q < KC; ++q) ccol[(size_t)q * nB + i] = q < cnt[i] ? tmp[(size_t)i * KSC + q] : g1 + i;
    // transpose slots for the single-reduction form: entry (i, k) at slot q
    // -> offset of entry (k, i); absent when the pattern is not symmetric
    std::vector<int> ctr((size_t)KC * nB);
    bool sym = true;
    for (int i = 0; i < nB && sym; ++i) {
      for (int q = 0; q < KC; ++q) {
        const size_t e = (size_t)q * nB + i;
        ctr[e] = (int)e;
        if (q >= cnt[i]) continue;
        const int kk = tmp[(size_t)i * KSC + q] - g1;
        const int* row = &tmp[(size_t)kk * KSC];
        const int* hit = std::lower_bound(row, row + cnt[kk], g1 + i);
        if (hit == row + cnt[kk] || *hit != g1 + i) { sym = false; break; }
        ctr[e] = (int)((size_t)(hit - row) * nB + kk);
      }
    }
    if (sym && (size_t)KC * nB <= (size_t)INT32_MAX) {
      CHK(S->alloc(&S->d_sctr, ctr.size()));
      CHK(S->alloc(&S->d_sst, (size_t)2 * n));
      CMS_CUDA(cudaMemcpyAsync(S->d_sctr, ctr.data(), ctr.size() * sizeof(int), cudaMemcpyHostToDevice, S->stream));
      S->sc_sym = 1;
    }
    CHK(S->alloc(&S->d_sccol, ccol.size()));
    CHK(S->alloc(&S->d_scoff, ccol.size()));
    CHK(S->alloc(&S->d_sccnt, (size_t)nB));
    CHK(S->alloc(&S->d_ssinv, (size_t)n));
    CHK(S->alloc(&S->d_sdep_ptr, (size_t)GRID_CAP + 1));
    CMS_CUDA(cudaMemcpyAsync(S->d_sccol, ccol.data(), ccol.size() * sizeof(int), cudaMemcpyHostToDevice, S->stream));
    CMS_CUDA(cudaMemcpyAsync(S->d_sccnt, cnt.data(), cnt.size(), cudaMemcpyHostToDevice, S->stream));
    CMS_CUDA(cudaStreamSynchronize(S->stream));
    S->sc_KC = KC;
    S->sc_nnz = nnz;
    S->sc_e0b = e0b;
    S->sc_tiles = 0;
    S->sc_state = 1;
  }
  if (S->sc_tiles == tiles) return CMS_OK;
  // neighbour tiles under Chat (tile t = natural cells [t n / nt, (t+1) n / nt))
  const int g1 = P.gstart[1], nB = n - g1;
  std::vector<int> ccol((size_t)S->sc_KC * nB);
  std::vector<signed char> cnt(nB);
  CMS_CUDA(cudaMemcpyAsync(ccol.data(), S->d_sccol, ccol.size() * sizeof(int), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaMemcpyAsync(cnt.data(), S->d_sccnt, cnt.size(), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  std::vector<int> tstart(tiles + 1);
  for (int t = 0; t <= tiles; ++t) tstart[t] = (int)((long long)t * n / tiles);
  std::vector<int> tile_nat(n);
  for (int t = 0; t < tiles; ++t)
    for (int c = tstart[t]; c < tstart[t + 1]; ++c) tile_nat[c] = t;
  std::vector<std::vector<int>> dep(tiles);
  auto add = [&](int a, int b) {
    for (int q : dep[a]) if (q == b) return;
    dep[a].push_back(b);
  };
  for (int i = 0; i < nB; ++i) {
    const int ti = tile_nat[P.perm[g1 + i]];
    for (int q = 0; q < cnt[i]; ++q) {
      const int tj = tile_nat[P.perm[ccol[(size_t)q * nB + i]]];
      if (tj != ti) { add(ti, tj); add(tj, ti); }
    }
  }
  std::vector<int> dptr(tiles + 1, 0), didx;
  for (int t = 0; t < tiles; ++t) {
    std::sort(dep[t].begin(), dep[t].end());
    didx.insert(didx.end(), dep[t].begin(), dep[t].end());
    dptr[t + 1] = (int)didx.size();
  }
  if (didx.size() + 1 > S->cap_sdep) {
    CHK(S->alloc(&S->d_sdep_idx, didx.size() + 1));
    S->cap_sdep = didx.size() + 1;
  }
  CMS_CUDA(cudaMemcpyAsync(S->d_sdep_ptr, dptr.data(), dptr.size() * sizeof(int), cudaMemcpyHostToDevice, S->stream));
  if (!didx.empty())
    CMS_CUDA(cudaMemcpyAsync(S->d_sdep_idx, didx.data(), didx.size() * sizeof(int), cudaMemcpyHostToDevice,
                             S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  S->sc_tiles = tiles;
  return CMS_OK;
}

// Chat's values and sinv from the FP32 matrix (once per solve).
static int schur_numeric(Solver* S) {
  const HostPattern& P = S->hp;
  const int n = P.n, g1 = P.gstart[1], nB = n - g1;
  const double nnz = (double)P.nnz_off;
  KLAUNCH(S, P_SCHUR_BUILD, 8.0 * nnz + 10.0 * n,
          (k_schur_diag<<<gsz(n), TPB, 0, S->stream>>>(n, g1, P.KL, S->d_col, S->d_nlo, S->d_nup, S->A32.aoff,
                                                         S->A32.diag, S->d_ssinv)));
  KLAUNCH(S, P_SCHUR_BUILD, 8.0 * nnz + 10.0 * n + 4.0 * n + 8.0 * (double)S->sc_nnz + nB,
          (k_schur_off<<<gsz(nB), TPB, 0, S->stream>>>(n, g1, nB, P.KL, S->sc_KC, S->d_col, S->d_nlo, S->d_nup,
                                                        S->A32.aoff, S->A32.diag, S->d_ssinv, S->d_sccol,
                                                        S->d_sccnt, S->d_scoff)));
  return CMS_OK;
}

// Algorithmic bytes of one reduced-system launch: the start (reduced
// right-hand side), per iteration P0 (8 vector accesses per row), A (p, r0,
// count, Chat, nu) and B (r, nu, r0, count, Chat, t), and the end (y update,
// x_B, then x_0 from b, 1/d and the group-0 rows' couplings).  Single-
// reduction form (sr): the start adds the transposed product (r0, count,
// Chat, transpose slots; f0, u, nu, p written), an iteration is X (s, t, y,
// p, nu, q, Chat; y, u, p, nu written) and Y (s, t, nu, u, r0, f0, Chat; q,
// s, t written), the end reads y, p, s.  Chat counts its stored couplings
// only (the kernel also reads the padding slots, which are not needed).
static double schur_bytes(const Solver* S, int iters, int sr) {
  const HostPattern& P = S->hp;
  const double n = P.n, g1 = P.gstart[1], nB = n - g1, C = 8.0 * (double)S->sc_nnz, E = 8.0 * (double)S->sc_e0b;
  if (sr) {
    const double start = 4.0 * n + 4.0 * g1 + E + nB + 12.0 * nB + (5.0 * nB + C + 4.0 * (double)S->sc_nnz + 16.0 * nB);
    const double it = (40.0 * nB + C) + (36.0 * nB + C);
    const double end = 20.0 * nB + 9.0 * g1 + E + 4.0 * nB + 4.0 * g1;
    return start + iters * it + end;
  }
  const double start = 4.0 * n + 4.0 * g1 + E + nB + 24.0 * nB;
  const double it = 32.0 * nB + (13.0 * nB + C) + (17.0 * nB + C);
  const double end = 24.0 * nB + 9.0 * g1 + E + 4.0 * nB + 4.0 * g1;
  return start + iters * it + end;
}

// Arguments of the reduced-system kernel for one system on `tiles` tiles.
static SchurArgs make_schur_args(Solver* S, int tiles, int maxit, double tol) {
  const HostPattern& P = S->hp;
  SchurArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = P.n; a.g1 = P.gstart[1]; a.nB = P.n - a.g1; a.KL = P.KL; a.G = P.G; a.KC = S->sc_KC;
  a.ntiles = tiles;
  a.toff = S->d_toff; a.dep_ptr = S->d_sdep_ptr; a.dep_idx = S->d_sdep_idx; a.progress = S->d_progress;
  a.ccol = S->d_sccol; a.coff = S->d_scoff; a.ccnt = S->d_sccnt;
  a.col = S->d_col; a.nlo = S->d_nlo; a.nup = S->d_nup; a.aoff = S->A32.aoff; a.sinv = S->d_ssinv;
  a.b = S->W32.b; a.x = S->W32.x;
  a.r = S->W32.r; a.r0 = S->W32.r0; a.p = S->W32.p; a.nu = S->W32.u; a.t = S->W32.v; a.y = S->W32.z;
  a.ctr = S->d_sctr; a.u = S->W32.vv[1]; a.q = S->W32.vv[2]; a.f0 = S->W32.vv[3];
  a.s_t = reinterpret_cast<float2*>(S->d_sst);
  a.yb = S->W32.vv[4];
  a.part = S->d_ppart; a.bar = &S->d_st->bar; a.st = S->d_st;
  a.maxit = maxit; a.tol = tol; a.spin_limit = kSpinLimit;
  return a;
}

// Layout of the reduced kernel for this handle (cms_solver_opts.reduced_layout,
// 0 = auto = 1024 threads x 2 rows in the single-reduction form, the fastest
// on the 1M systems) and the tiles it takes: its resident blocks on the
// device, at most one per 256 rows.  0 tiles when it cannot launch.
static int schur_layout_index(const Solver* S) {
  const int k = S->opts.reduced_layout;
  return (k >= 1 && k <= kSchurLayouts) ? k - 1 : 4;
}
// The layout that runs: a single-reduction layout needs a symmetric pattern
// of Chat; otherwise the three-phase layout of the same block and row shape.
static int schur_layout_run(const Solver* S) {
  const int k = schur_layout_index(S);
  const SchurLayout L = schur_layout(k);
  if (!L.sr || S->sc_sym) return k;
  for (int j = 0; j < kSchurLayouts; ++j) {
    const SchurLayout M = schur_layout(j);
    if (!M.sr && M.bs == L.bs) return j;
  }
  return 0;
}
static int schur_tiles(Solver* S, int layout) {
  const SchurLayout L = schur_layout(layout);
  int nsm = 0, per = 0, coop = 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, S->dev) != cudaSuccess || !coop ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, S->dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, L.single, L.bs, 0) != cudaSuccess || per <= 0) {
    cudaGetLastError();
    return 0;
  }
  return std::min(std::min(per * nsm, GRID_CAP), nblk(S->hp.n));
}

// The reduced FP32 inner solve (W32.b -> W32.x) as one cooperative launch.
static int run_schur_bicgstab(Solver* S, int tiles, int maxit, double tol) {
  SchurArgs a = make_schur_args(S, tiles, maxit, tol);
  const SchurLayout L = schur_layout(schur_layout_run(S));
  CMS_CUDA(cudaMemsetAsync(&S->d_st->bar, 0, sizeof(GridBar), S->stream));
  CMS_CUDA(cudaMemsetAsync(S->d_progress, 0, sizeof(unsigned int) * tiles * kProgressStride, S->stream));
  void* args[] = {&a};
  prof_begin(S);
  const cudaError_t e = cudaLaunchCooperativeKernel(L.single, dim3(tiles), dim3(L.bs), args, 0, S->stream);
  if (e != cudaSuccess) {
    std::snprintf(g_last_error, sizeof(g_last_error), "cooperative launch (reduced BiCGStab): %s",
                  cudaGetErrorString(e));
    return CMS_DEVICE_ERROR;
  }
  S->launches++;
  const size_t nrec = S->prof_recs.size();
  prof_end(S, P_SCHUR, 0.0);
  const bool recorded = S->prof_recs.size() > nrec;
  CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  if (S->h_st->bar.err) {
    std::snprintf(g_last_error, sizeof(g_last_error), "reduced BiCGStab: a grid barrier wait timed out");
    return CMS_DEVICE_ERROR;
  }
  if (recorded) S->prof_recs.back().bytes = schur_bytes(S, S->h_st->iter, L.sr);
  return CMS_OK;
}

// State of one system's refinement (run_refine's loop, shared with the
// ensembles' batched refinement).
struct RefineState {
  int steps = 0, inner_total = 0, maxit = 0, imax = 0, rmax = 0;
  double nrm0 = -1.0, prev = -1.0, rel = 1.0, tol = 0.0, itol = 0.0;
  cms_solve_info* info = nullptr;
};

// The FP64 residual of x64; go = false when the refinement ends (converged,
// capped or non-finite).  A correction that made the residual more than
// kRefineWorse times larger is undone (x64 -= the last correction, residual
// recomputed): worse = true.  BiCGStab's corrections are not monotone, so a
// small rise is kept; a failed inner solve raises it by orders of magnitude.
constexpr double kRefineWorse = 4.0;
static int refine_check(Solver* S, RefineState& R, bool& go, bool& worse) {
  const int n = S->hp.n;
  worse = false;
  CHK(resid64<double, double>(S, S->A64, S->W64.b, S->W64.x, S->W64.r, nullptr, S_NRM2));
  CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  double nrm = std::sqrt(S->h_st->s[S_NRM2]);
  if (R.steps > 0 && R.prev >= 0.0 && !(nrm <= kRefineWorse * R.prev)) {
    KLAUNCH(S, P_VEC, (double)n * 20, (k_ir_undo<<<gsz(n), TPB, 0, S->stream>>>(n, S->W32.x, S->W64.x, S->d_st)));
    CHK(resid64<double, double>(S, S->A64, S->W64.b, S->W64.x, S->W64.r, nullptr, S_NRM2));
    CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
    CMS_CUDA(cudaStreamSynchronize(S->stream));
    nrm = std::sqrt(S->h_st->s[S_NRM2]);
    worse = true;
  }
  if (R.nrm0 < 0) R.nrm0 = nrm;
  R.prev = nrm;
  R.rel = R.nrm0 > 0 ? nrm / R.nrm0 : 0.0;
  go = true;
  if (!std::isfinite(R.rel)) {
    R.info->status = CMS_NONFINITE;
    go = false;
  } else if (R.rel <= R.tol || R.steps >= R.rmax || R.inner_total >= R.maxit) {
    go = false;
  }
  return CMS_OK;
}

// Tolerance and iteration cap of the next inner FP32 solve.  By default
// (inner_tol and inner_max 0) the cap is the solve's remaining iteration
// budget and the tolerance asks the correction for what the outer residual
// still lacks, 0.5 tol / rel within [kInnerTolLo, kInnerTolHi]: one long inner
// solve takes a pressure-correction system to its tolerance, where short
// inner solves restarted from zero each lose the Krylov space built for the
// system's slow (smooth) modes and gain little (measured on the 1M-cell inlet
// flow: 89 % of the inner iterations of 50-iteration inner solves went to
// solves that ended unconverged at residual reductions of 0.05-0.9).  The
// floor 1e-6 lets a well-conditioned system (the velocity solves) reach a
// 1e-6 outer tolerance with one inner solve (1M-cell inlet flow step 4 %
// faster than with a 1e-5 floor, a 1M pressure-correction solve 1.62 ->
// 1.17 ms); the FP64 residual still decides convergence.
constexpr double kInnerTolLo = 1e-6, kInnerTolHi = 1e-3;
static void refine_inner_limits(const cms_solver_opts& o, RefineState& R) {
  const int left = std::max(1, R.maxit - R.inner_total);
  R.imax = o.inner_max > 0 ? std::min(o.inner_max, left) : left;
  R.itol = o.inner_tol > 0 ? o.inner_tol
                           : std::min(kInnerTolHi, std::max(kInnerTolLo, 0.5 * R.tol / std::max(R.rel, 1e-300)));
}

// Applies the inner solve's correction (W32.x, scaled by the residual norm).
static int refine_correct(Solver* S, RefineState& R) {
  const int n = S->hp.n;
  KLAUNCH(S, P_VEC, (double)n * 20, (k_ir_correct<<<gsz(n), TPB, 0, S->stream>>>(n, S->W32.x, S->W64.x, S->d_st)));
  ++R.steps;
  return CMS_OK;
}

// The rest of a refinement with the exact multicolour ILU(0) inner BiCGStab
// (or GMRES), from the current x64 and residual: the fallback of a reduced
// inner solve whose correction made the residual larger.
static int refine_exact(Solver* S, int nsolv, RefineState& R) {
  const int n = S->hp.n;
  S->cur_relax = 0;
  CHK(factor<float>(S, S->A32));
  ++S->reduced_fallbacks;
  bool go = true, worse = false;
  for (;;) {
    refine_inner_limits(S->opts, R);
    KLAUNCH(S, P_VEC, (double)n * 12, (k_ir_scale<<<gsz(n), TPB, 0, S->stream>>>(n, S->W64.r, S->W32.b, S->d_st)));
    if (nsolv == 3) {
      CHK(run_bicgstab<float>(S, S->A32, S->W32, R.imax, 2, R.itol, 1, false));
    } else {
      CMS_CUDA(cudaMemsetAsync(S->W32.x, 0, sizeof(float) * n, S->stream));
      CHK(run_gmres<float>(S, S->A32, S->W32, R.imax, R.itol, false));
    }
    CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
    CMS_CUDA(cudaStreamSynchronize(S->stream));
    R.inner_total += (nsolv == 3) ? S->h_st->iter : S->h_st->inner;
    if (S->h_st->nonfinite) break;
    CHK(refine_correct(S, R));
    CHK(refine_check(S, R, go, worse));
    if (!go || worse) break;
  }
  return CMS_OK;
}

static void refine_finish(RefineState& R) {
  R.info->iters = R.inner_total;
  R.info->inner = R.inner_total;
  R.info->refine_steps = R.steps;
  R.info->relres = R.rel;
  if (R.info->status == CMS_OK && R.rel > R.tol) R.info->status = CMS_NOT_CONVERGED;
}

// Iterative refinement: FP64 residual/correction, FP32 matrix + factor + Krylov.
static int run_refine(Solver* S, int nsolv, int maxit, double tol, cms_solve_info* info) {
  const HostPattern& P = S->hp;
  const int n = P.n;
  // A32 was written by the prologue; b64/x64 live in W64.b / W64.x.  The FP32
  // factor is the two-phase one when the persistent BiCGStab will run it.
  // inner_relax 2: the reduced system of cms_schur.cuh (any multicolour
  // ordering with an independent first group); 1: the two-phase factor
  // (more than two colours); 0: the exact multicolour ILU(0)
  const bool mc_persist = nsolv == 3 && S->opts.ordering == CMS_ORDER_MULTICOLOR && !S->opts.multi_kernel &&
                          persist_tiles(S) > 0;
  bool schur = mc_persist && S->opts.inner_relax == 2;
  if (schur) {  // the tiles of the reduced kernel's layout
    const int nt = schur_tiles(S, schur_layout_index(S));
    schur = nt > 0 && build_tiles(S, nt) == nt && schur_pattern(S, S->ptiles) == CMS_OK;
  }
  const bool relax = !schur && mc_persist && S->opts.inner_relax && P.G > 2;
  struct RelaxScope {  // the flags describe A32's factor and its solves only while this solve runs
    Solver* s;
    ~RelaxScope() { s->cur_relax = 0; s->cur_fuse = 0; }
  } relax_scope{S};
  S->cur_fuse = 1;
  if (schur) {
    CHK(schur_numeric(S));
  } else if (relax) {
    KLAUNCH(S, P_ILU0, (double)n * (3 * 4 + 2) + (double)(P.nnz_off) * (2 * 4 + 4),
            (k_ilu0_relax<float><<<gsz(n), TPB, 0, S->stream>>>(n, P.KL, P.gstart[1], S->d_col, S->d_nlo,
                                                                 S->d_nup, S->A32.aoff, S->A32.diag, S->A32.luoff,
                                                                 S->A32.invd)));
    S->cur_relax = 1;
  } else {
    CHK(factor<float>(S, S->A32));
  }
  RefineState R;
  R.info = info;
  R.tol = tol;
  R.maxit = maxit;
  R.rmax = S->opts.max_refine > 0 ? S->opts.max_refine : 30;
  for (;;) {
    bool go = true, worse = false;
    CHK(refine_check(S, R, go, worse));
    if (worse) {  // the last inner correction was no good
      if (go && (schur || relax)) CHK(refine_exact(S, nsolv, R));
      break;
    }
    if (!go) break;
    // inner FP32 solve A32 d = r/||r|| from d = 0 (factor already built)
    refine_inner_limits(S->opts, R);
    KLAUNCH(S, P_VEC, (double)n * 12, (k_ir_scale<<<gsz(n), TPB, 0, S->stream>>>(n, S->W64.r, S->W32.b, S->d_st)));
    if (schur) {
      CHK(run_schur_bicgstab(S, S->ptiles, R.imax, R.itol));  // tiles built above for its layout
    } else if (nsolv == 3) {
      CHK(run_bicgstab<float>(S, S->A32, S->W32, R.imax, 2, R.itol, 1, false));
    } else {
      CMS_CUDA(cudaMemsetAsync(S->W32.x, 0, sizeof(float) * n, S->stream));
      CHK(run_gmres<float>(S, S->A32, S->W32, R.imax, R.itol, false));
    }
    CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
    CMS_CUDA(cudaStreamSynchronize(S->stream));
    R.inner_total += (nsolv == 3) ? S->h_st->iter : S->h_st->inner;
    // an FP32 inner solve that overflowed (a near-breakdown of its recurrence)
    // gives no correction: with the reduced or two-phase form the rest runs
    // on the exact factor, else the refinement ends with the FP64 iterate
    if (S->h_st->nonfinite) {
      if (schur || relax) CHK(refine_exact(S, nsolv, R));
      break;
    }
    CHK(refine_correct(S, R));
  }
  refine_finish(R);
  return CMS_OK;
}

// The whole solve() on device-resident natural-order arrays.
template <typename T>
static int solve_dev(Solver* S, const T* acoef, T* ss, const T* sp, T* res, T* phi, T relax, int nswp, int nsolv,
                     cms_solve_info* info, int nvar = 0) {
  const HostPattern& P = S->hp;
  cms_solve_info loc{};
  if (!info) info = &loc;
  std::memset(info, 0, sizeof(*info));
  info->ncolors = P.G;
  info->true_relres = -1.0;
  if (nsolv < 0 || nsolv > 8) return info->status = CMS_UNSUPPORTED;
  const bool legacy = nsolv != 3 && nsolv != 4;
  if (nsolv >= 6) {
    const int props = legacy_props(S);
    if (props < 0) return info->status = CMS_DEVICE_ERROR;
    const int kind = legacy_plan(nsolv, nvar, 0.0, nswp, S->opts.nswp0_vel).kind;
    if (!(props & LEG_FIVE_POINT)) {
      std::snprintf(g_last_error, sizeof(g_last_error),
                    "nsolv %d: the 5-point solvers need exactly four faces (N, E, S, W) per cell", nsolv);
      return info->status = CMS_UNSUPPORTED;
    }
    if (kind == LK_SIP && !(props & LEG_SIP_ORDER)) {
      std::snprintf(g_last_error, sizeof(g_last_error),
                    "nsolv %d: SIP runs in the natural ordering of a grid numbered row by row from the south-west",
                    nsolv);
      return info->status = CMS_UNSUPPORTED;
    }
  }
  const int maxit = S->opts.max_iters > 0 ? S->opts.max_iters : nswp;
  const double tol = S->opts.tol > 0 ? S->opts.tol : 1e-3;
  const int norm = S->opts.norm == 2 ? 2 : 1;
  int prec = S->opts.precision;
  if (sizeof(T) == 4 || legacy) prec = sizeof(T) == 4 ? CMS_PREC_FP32 : CMS_PREC_FP64;
  const bool is64 = sizeof(T) == 8;
  Mat<T>& A = *reinterpret_cast<Mat<T>*>(is64 ? (void*)&S->A64 : (void*)&S->A32);
  Work<T>& W = *reinterpret_cast<Work<T>*>(is64 ? (void*)&S->W64 : (void*)&S->W32);
  // prologue: ap, ss, res, rmom + device-order system (and FP32 copy)
  float* a2 = (is64 && prec == CMS_PREC_FP32_REFINE) ? S->A32.aoff : nullptr;
  float* d2 = (is64 && prec == CMS_PREC_FP32_REFINE) ? S->A32.diag : nullptr;
  {
    const double sz = sizeof(T);
    const double per = P.nmf * (sz + 4 + 1) + 4 + 4 + 4 + sz * 7 + (a2 ? 4 : 0);
    KLAUNCH(S, P_PROLOGUE, (double)P.n * per + (double)P.nnz_off * (sz + (a2 ? 4 : 0)),
            (k_prologue<T, float><<<gsz(P.n), TPB, 0, S->stream>>>(P.n, P.nmf, acoef, ss, sp, res, phi, S->d_c2c,
                                                                     S->d_ncface, S->d_iwet, S->d_fslot, S->d_iperm,
                                                                     relax, A.aoff, A.diag, W.b, W.x, a2, d2,
                                                                     S->d_part, S->d_st)));
  }
  if (S->opts.verify) {
    if (is64) CHK((resid64<double, double>(S, S->A64, S->W64.b, S->W64.x, nullptr, nullptr, S_TRUE0)));
    else {
      KLAUNCH(S, P_VEC, (double)P.n * 12,
              (k_convert<double, float><<<gsz(P.n), TPB, 0, S->stream>>>(P.n, S->W32.b, S->W64.r)));
      CHK((resid64<float, float>(S, S->A32, S->W64.r, S->W32.x, nullptr, nullptr, S_TRUE0)));
    }
  }
  LegPlan plan;
  int leg_sweeps = 0;
  if (legacy) {
    double rm = 0.0;
    if (nsolv == 2 || nsolv == 5) {  // the branch reads this call's rmom
      CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
      CMS_CUDA(cudaStreamSynchronize(S->stream));
      rm = S->h_st->s[S_RMOM];
    }
    plan = legacy_plan(nsolv, nvar, rm, maxit, S->opts.nswp0_vel);
  }
  if (plan.kind == LK_NONE) {
  } else if (plan.kind == LK_GS) {
    CHK(run_gauss_seidel<T>(S, A, W, plan.sweeps, plan.symmetric, plan.sor, S->opts.relaxsor, &leg_sweeps));
  } else if (plan.kind == LK_SIP) {
    CHK(run_sip<T>(S, A, W, acoef, maxit));
  } else if (plan.kind == LK_ICCG) {
    CHK(run_iccg<T>(S, A, W, maxit));
  } else if (plan.kind == LK_ICCGSTAB) {
    CHK(run_iccgstab<T>(S, A, W, maxit));
  } else if (is64 && prec == CMS_PREC_FP32_REFINE) {
    CHK(run_refine(S, legacy ? 3 : nsolv, maxit, tol, info));
  } else {
    CHK(run_krylov<T>(S, A, W, legacy ? 3 : nsolv, maxit, norm, tol, 0));
  }
  if (S->opts.verify) {
    if (is64) CHK((resid64<double, double>(S, S->A64, S->W64.b, S->W64.x, nullptr, nullptr, S_TRUE1)));
    else CHK((resid64<float, float>(S, S->A32, S->W64.r, S->W32.x, nullptr, nullptr, S_TRUE1)));
  }
  KLAUNCH(S, P_VEC, (double)P.n * (4 + 2 * sizeof(T)),
          (k_scatter<T, T><<<gsz(P.n), TPB, 0, S->stream>>>(P.n, S->d_perm, W.x, phi)));
  CMS_CUDA(cudaMemcpyAsync(S->h_st, S->d_st, sizeof(DevState), cudaMemcpyDeviceToHost, S->stream));
  CMS_CUDA(cudaStreamSynchronize(S->stream));
  const DevState& h = *S->h_st;
  info->rmom = h.s[S_RMOM];
  if (plan.kind == LK_GS || plan.kind == LK_NONE) {
    info->iters = info->inner = leg_sweeps;  // fixed sweep count, no stopping test
  } else if (!(is64 && prec == CMS_PREC_FP32_REFINE)) {
    info->iters = h.iter;
    info->inner = (nsolv == 4) ? h.inner : h.iter;
    info->relres = h.s[S_RELRES];
    if (h.nonfinite) info->status = CMS_NONFINITE;
    else if (!h.converged) info->status = CMS_NOT_CONVERGED;
  }
  if (S->opts.verify) {
    const double t0 = std::sqrt(h.s[S_TRUE0]), t1 = std::sqrt(h.s[S_TRUE1]);
    info->true_relres = t0 > 0 ? t1 / t0 : 0.0;
    if (!std::isfinite(t1)) info->status = CMS_NONFINITE;
  }
  return info->status;
}

template <typename T>
static int solve_host(Solver* S, const T* acoef, T* ss, const T* sp, T* res, T* phi, T relax, int nswp, int nsolv,
                      cms_solve_info* info, int nvar = 0) {
  const bool is64 = sizeof(T) == 8;
  Staging<T>& st = *reinterpret_cast<Staging<T>*>(is64 ? (void*)&S->S64 : (void*)&S->S32);
  CHK(alloc_staging<T>(S, st));
  const size_t nD = S->hp.nD, nmf = S->hp.nmf;
  cudaStream_t s = S->stream;
  CMS_CUDA(cudaMemcpyAsync(st.acoef, acoef, nD * nmf * sizeof(T), cudaMemcpyHostToDevice, s));
  CMS_CUDA(cudaMemcpyAsync(st.ss, ss, nD * sizeof(T), cudaMemcpyHostToDevice, s));
  CMS_CUDA(cudaMemcpyAsync(st.sp, sp, nD * sizeof(T), cudaMemcpyHostToDevice, s));
  CMS_CUDA(cudaMemcpyAsync(st.phi, phi, nD * sizeof(T), cudaMemcpyHostToDevice, s));
  const int rc = solve_dev<T>(S, st.acoef, st.ss, st.sp, st.res, st.phi, relax, nswp, nsolv, info, nvar);
  if (rc == CMS_DEVICE_ERROR || rc == CMS_BAD_ARGUMENT || rc == CMS_UNSUPPORTED) return rc;
  const size_t n = S->hp.n;
  CMS_CUDA(cudaMemcpyAsync(ss, st.ss, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  CMS_CUDA(cudaMemcpyAsync(res, st.res, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  CMS_CUDA(cudaMemcpyAsync(phi, st.phi, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  CMS_CUDA(cudaStreamSynchronize(s));
  return rc;
}

}  // namespace cms

using cms::Solver;

extern "C" {

void cms_solver_default_opts(cms_solver_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->ordering = CMS_ORDER_MULTICOLOR;
  o->precision = CMS_PREC_FP64;
  o->norm = 1;
  o->tol = 1.0e-3;
  o->max_iters = 0;
  o->inner_tol = 0.0;
  o->inner_max = 0;
  o->max_refine = 30;
  o->verify = 1;
  o->multi_kernel = 0;
  o->inner_relax = 2;
  o->relaxsor = 1.8;   // flow.F90:131
  o->nswp0_vel = 5;    // nswp0(2) of the hybrid solver's defaults (flow.F90:795-798)
}

int cms_solver_create(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface,
                      const int* iwet, const cms_solver_opts* opts, cms_solver** out) {
  if (!out) return CMS_BAD_ARGUMENT;
  return cms::create(ncells, ncellsD, nmaxfaces, cell2cell, ncface, iwet, opts, out);
}

int cms_solver_update_wet(cms_solver* s, const int* iwet) {
  if (!s || !iwet) return CMS_BAD_ARGUMENT;
  if (cudaMemcpyAsync(s->d_iwet, iwet, s->hp.nD * sizeof(int), cudaMemcpyHostToDevice, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess)
    return CMS_DEVICE_ERROR;
  return CMS_OK;
}

int cms_solver_set_tiles(cms_solver* s, int tiles) {
  if (!s || tiles < 0) return -CMS_BAD_ARGUMENT;
  const int cap = cms::persist_capacity(s->dev);
  if (cap <= 0) return -CMS_UNSUPPORTED;
  const int nt = cms::build_tiles(s, tiles == 0 ? std::min(cap, cms::nblk(s->hp.n)) : std::min(tiles, cap));
  return nt > 0 ? nt : -CMS_UNSUPPORTED;
}

int cms_solver_set_opts(cms_solver* s, const cms_solver_opts* o) {
  if (!s || !o) return CMS_BAD_ARGUMENT;
  if (o->ordering != s->opts.ordering) return CMS_BAD_ARGUMENT;  // the ordering is fixed at creation
  s->opts = *o;
  return CMS_OK;
}

int cms_solver_solve_d(cms_solver* s, const double* acoef, double* ss, const double* sp, double* res, double* phi,
                       double relax, int nswp, int nsolv, cms_solve_info* info) {
  if (!s || !acoef || !ss || !sp || !res || !phi) return CMS_BAD_ARGUMENT;
  return cms::solve_host<double>(s, acoef, ss, sp, res, phi, relax, nswp, nsolv, info);
}
int cms_solver_solve_f(cms_solver* s, const float* acoef, float* ss, const float* sp, float* res, float* phi,
                       float relax, int nswp, int nsolv, cms_solve_info* info) {
  if (!s || !acoef || !ss || !sp || !res || !phi) return CMS_BAD_ARGUMENT;
  return cms::solve_host<float>(s, acoef, ss, sp, res, phi, relax, nswp, nsolv, info);
}
int cms_solver_solve_dev_d(cms_solver* s, const double* acoef, double* ss, const double* sp, double* res,
                           double* phi, double relax, int nswp, int nsolv, cms_solve_info* info) {
  if (!s || !acoef || !ss || !sp || !res || !phi) return CMS_BAD_ARGUMENT;
  return cms::solve_dev<double>(s, acoef, ss, sp, res, phi, relax, nswp, nsolv, info);
}
int cms_solver_solve_dev_f(cms_solver* s, const float* acoef, float* ss, const float* sp, float* res, float* phi,
                           float relax, int nswp, int nsolv, cms_solve_info* info) {
  if (!s || !acoef || !ss || !sp || !res || !phi) return CMS_BAD_ARGUMENT;
  return cms::solve_dev<float>(s, acoef, ss, sp, res, phi, relax, nswp, nsolv, info);
}

int cms_solver_solve_n_d(cms_solver* s, int n, const double* acoef, double* ss, const double* sp, double* res,
                         double* phi, double relax, int nswp, int nsolv, cms_solve_info* info) {
  if (!s || !acoef || !ss || !sp || !res || !phi) return CMS_BAD_ARGUMENT;
  return cms::solve_host<double>(s, acoef, ss, sp, res, phi, relax, nswp, nsolv, info, n);
}
int cms_solver_solve_n_f(cms_solver* s, int n, const float* acoef, float* ss, const float* sp, float* res, float* phi,
                         float relax, int nswp, int nsolv, cms_solve_info* info) {
  if (!s || !acoef || !ss || !sp || !res || !phi) return CMS_BAD_ARGUMENT;
  return cms::solve_host<float>(s, acoef, ss, sp, res, phi, relax, nswp, nsolv, info, n);
}
int cms_solver_solve_dev_n_d(cms_solver* s, int n, const double* acoef, double* ss, const double* sp, double* res,
                             double* phi, double relax, int nswp, int nsolv, cms_solve_info* info) {
  if (!s || !acoef || !ss || !sp || !res || !phi) return CMS_BAD_ARGUMENT;
  return cms::solve_dev<double>(s, acoef, ss, sp, res, phi, relax, nswp, nsolv, info, n);
}
int cms_solver_solve_dev_n_f(cms_solver* s, int n, const float* acoef, float* ss, const float* sp, float* res,
                             float* phi, float relax, int nswp, int nsolv, cms_solve_info* info) {
  if (!s || !acoef || !ss || !sp || !res || !phi) return CMS_BAD_ARGUMENT;
  return cms::solve_dev<float>(s, acoef, ss, sp, res, phi, relax, nswp, nsolv, info, n);
}

int cms_solver_profile(cms_solver* s, int enable) {
  if (!s) return CMS_BAD_ARGUMENT;
  s->prof_on = enable ? 1 : 0;
  return CMS_OK;
}

int cms_solver_profile_read(cms_solver* s, int reset, double* ms, double* bytes, long long* count) {
  if (!s) return CMS_BAD_ARGUMENT;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return CMS_DEVICE_ERROR;
  for (const auto& r : s->prof_recs) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, s->ev_pool[r.ev], s->ev_pool[r.ev + 1]) != cudaSuccess) return CMS_DEVICE_ERROR;
    s->prof_ms[r.cat] += t;
    s->prof_bytes[r.cat] += r.bytes;
    s->prof_count[r.cat] += 1;
  }
  s->prof_recs.clear();
  s->ev_used = 0;
  for (int c = 0; c < cms::P_NCAT; ++c) {
    if (ms) ms[c] = s->prof_ms[c];
    if (bytes) bytes[c] = s->prof_bytes[c];
    if (count) count[c] = s->prof_count[c];
    if (reset) { s->prof_ms[c] = 0; s->prof_bytes[c] = 0; s->prof_count[c] = 0; }
  }
  return CMS_OK;
}

int cms_solver_ncolors(const cms_solver* s) { return s ? s->hp.G : -1; }
size_t cms_solver_device_bytes(const cms_solver* s) { return s ? s->bytes : 0; }
int cms_solver_get_perm(const cms_solver* s, int* perm) {
  if (!s || !perm) return CMS_BAD_ARGUMENT;
  std::memcpy(perm, s->hp.perm.data(), s->hp.perm.size() * sizeof(int));
  return CMS_OK;
}
long long cms_solver_launches(const cms_solver* s) { return s ? s->launches : 0; }
void* cms_solver_stream(cms_solver* s) { return s ? (void*)s->stream : nullptr; }

void cms_solver_destroy(cms_solver* s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (void* p : s->allocs) cudaFree(p);
  for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
  if (s->h_st) cudaFreeHost(s->h_st);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

long long cms_solver_refine_fallbacks(const cms_solver* s) { return s ? s->reduced_fallbacks : 0; }

// ---- reference-shaped global API ----
static cms_solver* g_solver = nullptr;
static cms_solver_opts g_opts;
static bool g_opts_set = false;
static cms_solve_info g_info;
static std::mutex g_mu;

int cms_gpu_init(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface, const int* iwet) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_solver) { cms_solver_destroy(g_solver); g_solver = nullptr; }
  if (!g_opts_set) cms_solver_default_opts(&g_opts);
  return cms_solver_create(ncells, ncellsD, nmaxfaces, cell2cell, ncface, iwet, &g_opts, &g_solver);
}
int cms_gpu_set_opts(const cms_solver_opts* o) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!o) return CMS_BAD_ARGUMENT;
  if (g_solver && o->ordering != g_opts.ordering) return CMS_BAD_ARGUMENT;
  g_opts = *o;
  g_opts_set = true;
  if (g_solver) return cms_solver_set_opts(g_solver, o);
  return CMS_OK;
}
int cms_gpu_update_wet(const int* iwet) {
  std::lock_guard<std::mutex> lk(g_mu);
  return g_solver ? cms_solver_update_wet(g_solver, iwet) : CMS_BAD_ARGUMENT;
}
int cms_gpu_solve_d(int n, const double* acoef, double* ss, const double* sp, double* res, double* phi, double relax,
                    int nswp, int nsolv, double* rmom) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_solver) return CMS_BAD_ARGUMENT;
  int rc = cms_solver_solve_n_d(g_solver, n, acoef, ss, sp, res, phi, relax, nswp, nsolv, &g_info);
  if (rmom) *rmom = g_info.rmom;
  return rc;
}
int cms_gpu_solve_f(int n, const float* acoef, float* ss, const float* sp, float* res, float* phi, float relax,
                    int nswp, int nsolv, float* rmom) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_solver) return CMS_BAD_ARGUMENT;
  int rc = cms_solver_solve_n_f(g_solver, n, acoef, ss, sp, res, phi, relax, nswp, nsolv, &g_info);
  if (rmom) *rmom = (float)g_info.rmom;
  return rc;
}
int cms_gpu_last_info(cms_solve_info* info) {
  if (!info) return CMS_BAD_ARGUMENT;
  *info = g_info;
  return CMS_OK;
}
int cms_gpu_finalize(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_solver) { cms_solver_destroy(g_solver); g_solver = nullptr; }
  return CMS_OK;
}

int cms_order_build(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell, const int* ncface, int ordering,
                    int* perm, int* gstart, int* kl_ku) {
  if (!cell2cell || !ncface || !perm || !gstart || !kl_ku) return -CMS_BAD_ARGUMENT;
  cms::HostPattern P;
  std::string err = cms::build_pattern(ncells, ncellsD, nmaxfaces, cell2cell, ncface, ordering, P);
  if (!err.empty()) {
    std::snprintf(g_last_error, sizeof(g_last_error), "%s", err.c_str());
    return -CMS_BAD_ARGUMENT;
  }
  std::memcpy(perm, P.perm.data(), sizeof(int) * P.n);
  std::memcpy(gstart, P.gstart.data(), sizeof(int) * (P.G + 1));
  kl_ku[0] = P.KL;
  kl_ku[1] = P.KU;
  return P.G;
}

const char* cms_gpu_version(void) { return "cmsgpu 0.1 (sm_100a)"; }

int cms_solver_persist_wait_selftest(cms_solver* s, unsigned int spin_limit, int which) {
  if (!s || spin_limit == 0 || (which != 0 && which != 1)) return CMS_BAD_ARGUMENT;
  return cms::persist_wait_selftest(s, spin_limit, which);
}

int cms_solver_wait_selftest(cms_solver* s, unsigned int spin_limit) {
  if (!s || spin_limit == 0) return CMS_BAD_ARGUMENT;
  return cms::pipe_wait_selftest(s, spin_limit);
}

const char* cms_gpu_last_error(void) { return g_last_error; }

}  // extern "C"

// The device flow step shares this translation unit (and the handle internals).
#include "cms_flow_host.cuh"
#include "cms_ensemble_host.cuh"
#include "cms_adjoint_host.cuh"
