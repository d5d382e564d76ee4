// Persistent ILU(0)-BiCGStab: one cooperative launch runs the start and every
// iteration of a solve (pbicgstab.f90:20-96) on a factor built beforehand
// (k_ilu0).  No host round trip happens inside a solve.
//
// Work split.  Each block owns one tile: a contiguous range of natural cell
// numbers.  Inside a colour group the device rows keep natural order, so the
// rows of tile t in group g are one contiguous device range
// toff[g][t] .. toff[g][t+1].  Every phase (one group of a sweep, an SpMV,
// an update) runs over the block's own rows only.
//
// Ordering between phases.  Rows of a tile are coupled only to rows of a few
// neighbouring tiles (dep lists, built on the host from the pattern, and
// symmetric).  Each block publishes how many phases it has completed
// (progress[t * kProgressStride], a release store after every phase; one
// counter per 128-byte line, so that a tile's stores do not disturb the line
// other tiles are polling for their neighbours); before a phase in which
// it has rows, it waits until every neighbour has completed all earlier
// phases (acquire loads).  So a block reads neighbour values only after they
// are written, and a neighbour never writes its rows of a phase while this
// block may still read their previous values (it would first wait for this
// block).  No grid-wide barrier is needed inside the triangular sweeps.
//
// Dot products: every block writes its partial sums, passes a grid-wide
// barrier (a monotone arrival counter), then sums all partials itself in a
// fixed order, so all blocks hold the same value and take the same branch;
// the result does not depend on timing.  Partials are double-buffered.
//
// Every wait is bounded: after kSpinLimit polls the block records an error in
// the barrier state, every later wait returns at once, and the kernel ends;
// the host reports CMS_DEVICE_ERROR.  The launch is cooperative, so all
// blocks are resident and every wait can be satisfied.
//
// Arrays written inside the launch are read after an acquire (a neighbour
// wait or a grid barrier, by the block's waiting thread) and a block barrier,
// so the PTX memory model orders the writers' stores before those reads, as
// after a grid.sync(); the reads are ordinary L1-allocating loads: rows next
// to each other gather from the same lines, so many gathers hit in L1 (against
// L2-only loads: +8 % on the 1M-cell inlet flow step with FP32 refinement,
// the FP64 drop-in equal, the same iterates).  Partial sums, read once after
// a barrier, stay L2-only.
//
// Two-phase preconditioner (relax = 1, the FP32 solve inside iterative
// refinement): groups 1..G-1 are treated as one group.  The factor is ILU(0)
// of A with the couplings among rows of groups >= 1 removed (k_ilu0_relax):
// a multicolour grid that needs more than two colours (telescoping
// interfaces) then sweeps like a red/black one, two phases forward and one
// backward, while the SpMV keeps every coupling of A.  Only a few interface
// couplings are dropped; the refinement's FP64 residual makes the result
// independent of that choice.
#pragma once
#include "cms_common.cuh"

namespace cms {

constexpr int kProgressStride = 32;  // unsigned ints between two tiles' progress counters (128 bytes)
constexpr int NSMAX = 9;  // sums per reduction (partial-sum buffer stride)

__device__ __forceinline__ void red_release_add(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename T>
__device__ __forceinline__ T ldm(const T* p) { return __ldca(p); }  // load of data written in this launch

template <typename T>
struct PersistArgs {
  int n, KL, KU, G;
  int klB, kuB;            // slot bounds over groups 1..G-1
  int gku_last;            // upper slots of the last group (0: its backward step is fused)
  int spmv0;               // 1: group 0 has no lower couplings and its own backward
                           // phase; the SpMV of its rows is done in that phase
  int relax;               // 1: two-phase preconditioner (factor from k_ilu0_relax)
  int fuse_upd;            // 1 (L2 stopping test only): the x/r update is done in the next
                           // iteration's forward phases, its sums come from identities
  int g1;                  // first row of group 1
  const int* gkl;          // [G] lower slots per group
  const int* gku;          // [G] upper slots per group
  int ntiles;              // tiles (blocks) of this system
  int tile;                // this block's tile (set in the block's own copy)
  const int* toff;         // [G][ntiles+1] tile row ranges per group
  const int* dep_ptr;      // [ntiles+1]
  const int* dep_idx;      // neighbour tiles of each tile
  unsigned int* progress;  // [ntiles * kProgressStride] phases completed per tile (zero at launch)
  const int* col;
  const signed char* nlo;
  const signed char* nup;
  const T* aoff;
  const T* diag;
  const T* luoff;
  const T* invd;
  const T* b;
  T* x;
  T* r;
  T* r0;
  T* p;
  T* u;
  T* v;
  T* z;
  double* part;  // [2][NSMAX][ntiles]
  GridBar* bar;  // count: barrier arrivals (zero at launch); err: a wait gave up
  DevState* st;
  int maxit, norm, xzero;
  double tol;
  unsigned int spin_limit;  // polls before a wait gives up (kSpinLimit; smaller in the wait self-test)
};

// Per-block phase state (uniform across the block).
struct PhaseState {
  unsigned int done;    // phases this block has completed
  unsigned int target;  // barrier arrivals that release the next grid barrier
  bool fresh;           // just passed a grid barrier: every tile is in step
  bool ok;              // no wait has given up
};

__device__ __forceinline__ bool bar_failed(GridBar* b) { return *(volatile int*)&b->err != 0; }

// Waits until every neighbour tile has completed ph.done phases.  (These
// helpers take any argument struct with the tile, dependency, progress,
// barrier and partial-sum fields of PersistArgs.)
template <class Args>
__device__ __forceinline__ void wait_neighbours(const Args& A, PhaseState& ph) {
  __shared__ int s_fail;
  if (ph.fresh) { ph.fresh = false; return; }
  if (threadIdx.x < 32) {
    int fail = 0;
    const int d0 = A.dep_ptr[A.tile], d1 = A.dep_ptr[A.tile + 1];
    for (int i = d0 + (int)threadIdx.x; i < d1 && !fail; i += 32) {
      const unsigned int* f = A.progress + (size_t)A.dep_idx[i] * kProgressStride;
      unsigned int spins = 0;
      while (ld_acquire(f) < ph.done) {
        if (++spins > A.spin_limit) { atomicExch(&A.bar->err, 1); fail = 1; break; }
        if ((spins & 255u) == 0 && bar_failed(A.bar)) { fail = 1; break; }
      }
    }
    fail = __any_sync(0xffffffffu, fail);
    if (threadIdx.x == 0) s_fail = fail;
  }
  __syncthreads();
  if (s_fail) ph.ok = false;
}

// Ends a phase: publishes the completed count.
template <class Args>
__device__ __forceinline__ void end_phase(const Args& A, PhaseState& ph) {
  __syncthreads();
  ++ph.done;
  ph.fresh = false;
  if (threadIdx.x == 0) st_release(A.progress + (size_t)A.tile * kProgressStride, ph.done);
}

// Grid-wide barrier on a monotone arrival counter.
template <class Args>
__device__ __forceinline__ void grid_barrier(const Args& A, PhaseState& ph) {
  __shared__ int s_fail;
  __syncthreads();
  ph.target += A.ntiles;
  if (threadIdx.x == 0) {
    int fail = 0;
    if (bar_failed(A.bar)) {
      fail = 1;
    } else {
      red_release_add(&A.bar->count, 1u);
      unsigned int spins = 0;
      while (ld_acquire(&A.bar->count) < ph.target) {
        if (++spins > A.spin_limit) { atomicExch(&A.bar->err, 1); fail = 1; break; }
        if ((spins & 255u) == 0 && bar_failed(A.bar)) { fail = 1; break; }
      }
    }
    s_fail = fail;
  }
  __syncthreads();
  if (s_fail) ph.ok = false;
  ph.fresh = true;
}

// Writes this block's partial sums of NS values into buffer buf.
template <int NS, class Args>
__device__ __forceinline__ void put_partials(const Args& A, double (&v)[NS], int buf) {
  block_sum<NS>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NS; ++q) A.part[((size_t)buf * NSMAX + q) * A.ntiles + A.tile] = v[q];
  }
}

// After a grid barrier: every thread of every block gets the grid totals.
template <int NS, class Args>
__device__ __forceinline__ void get_totals(const Args& A, double (&tot)[NS], int buf) {
  __shared__ double bc[NS];
  double acc[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    acc[q] = 0.0;
    for (int bb = threadIdx.x; bb < A.ntiles; bb += blockDim.x)
      acc[q] += __ldcg(&A.part[((size_t)buf * NSMAX + q) * A.ntiles + bb]);
  }
  block_sum<NS>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NS; ++q) bc[q] = acc[q];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NS; ++q) tot[q] = bc[q];
  __syncthreads();
}

// Rows of this block's tile in group g.
template <typename T>
__device__ __forceinline__ int2 tile_rows(const PersistArgs<T>& A, int g) {
  const int* o = A.toff + (size_t)g * (A.ntiles + 1) + A.tile;
  return make_int2(__ldg(o), __ldg(o + 1));
}

// Rows [r0, r1) of a phase, NR rows per thread at a time (r, r + TPB, ...),
// so that each thread has the loads of NR rows in flight together: every
// phase body issues all loads of a batch before its first store.  Rows past
// r1 are replaced by the first row of the batch (loads stay in bounds) and
// marked !ok; their results are not stored.
template <typename T>
constexpr int NRT = 2;  // rows per thread per batch (register budget; measured best for FP32 and FP64)
template <int NR, typename F>
__device__ __forceinline__ void for_rows(int r0, int r1, F&& f) {
  for (int base = r0 + (int)threadIdx.x; base < r1; base += NR * (int)blockDim.x) {
    int r[NR];
    bool ok[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) {
      r[q] = base + q * (int)blockDim.x;
      ok[q] = r[q] < r1;
      if (!ok[q]) r[q] = base;
    }
    f(r, ok);
  }
}

// Rows of this tile in groups ga..gb as one index space, so that small groups
// do not each cost a batch of their own.  With up to GFLAT groups the tile's
// ranges sit in shared memory (s_lo: first row of each group's range, s_pre:
// prefix counts); with more groups (level schedules) each group is a loop.
constexpr int GFLAT = 16;
template <int NR, typename T, typename F>
__device__ __forceinline__ void for_rows_g(const PersistArgs<T>& A, const int* s_lo, const int* s_pre, int ga, int gb,
                                           F&& f) {
  if (A.G > GFLAT) {
    for (int g = ga; g <= gb; ++g) {
      const int2 rr = tile_rows(A, g);
      for_rows<NR>(rr.x, rr.y, f);
    }
    return;
  }
  const int k0 = s_pre[ga], k1 = s_pre[gb + 1];
  for (int base = k0 + (int)threadIdx.x; base < k1; base += NR * (int)blockDim.x) {
    int r[NR];
    bool ok[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) {
      int k = base + q * (int)blockDim.x;
      ok[q] = k < k1;
      if (!ok[q]) k = base;
      int g = ga;
      while (g < gb && k >= s_pre[g + 1]) ++g;
      r[q] = s_lo[g] + (k - s_pre[g]);
    }
    f(r, ok);
  }
}

// rows of this tile in groups ga..gb
template <typename T>
__device__ __forceinline__ int tile_count(const PersistArgs<T>& A, const int* s_pre, int ga, int gb) {
  if (A.G <= GFLAT) return s_pre[gb + 1] - s_pre[ga];
  int c = 0;
  for (int g = ga; g <= gb; ++g) {
    const int2 rr = tile_rows(A, g);
    c += rr.y - rr.x;
  }
  return c;
}

// Slot sums over NR rows at once, slot loops bounded by the group's slot
// count (uniform) and each term predicated on the row's own count, so padding
// slots cost no memory traffic.  Terms are applied one by one in slot order
// (the order of k_fwd / k_bwd / k_spmv, so both paths round alike).

// acc - sum_{lower} l_rj w_j over couplings to rows j < cmax (in the
// two-phase preconditioner the others are not part of the factor and are not
// read)
template <typename T, int NR>
__device__ __forceinline__ void lower_sub(const PersistArgs<T>& A, T (&acc)[NR], const T* w, const int (&r)[NR],
                                          int klg, int cmax = 0x7fffffff) {
  int kl[NR];
#pragma unroll
  for (int q = 0; q < NR; ++q) kl[q] = __ldg(&A.nlo[r[q]]);
#pragma unroll
  for (int s = 0; s < KMAX; ++s) {
    if (s < klg) {
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        const size_t e = (size_t)s * A.n + r[q];
        const int c = __ldg(&A.col[e]);
        if (s < kl[q] && c < cmax) acc[q] = acc[q] - __ldg(&A.luoff[e]) * ldm(&w[c]);
      }
    }
  }
}
// acc - sum_{upper} u_rk w_k
template <typename T, int NR>
__device__ __forceinline__ void upper_sub(const PersistArgs<T>& A, T (&acc)[NR], const T* w, const int (&r)[NR],
                                          int kug) {
  int ku[NR];
#pragma unroll
  for (int q = 0; q < NR; ++q) ku[q] = __ldg(&A.nup[r[q]]);
#pragma unroll
  for (int t = 0; t < KMAX; ++t) {
    if (t < kug) {
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        const size_t e = (size_t)(A.KL + t) * A.n + r[q];
        if (t < ku[q]) acc[q] = acc[q] - __ldg(&A.luoff[e]) * ldm(&w[__ldg(&A.col[e])]);
      }
    }
  }
}
// sum_{all} a_rj w_j (lower slots, then upper slots) for rows of a group
// with slot bounds klg, kug
template <typename T, int NR>
__device__ __forceinline__ void offdiag_sum(const PersistArgs<T>& A, T (&acc)[NR], const T* w, const int (&r)[NR],
                                            int klg, int kug) {
  int kl[NR], ku[NR];
#pragma unroll
  for (int q = 0; q < NR; ++q) {
    kl[q] = __ldg(&A.nlo[r[q]]);
    ku[q] = __ldg(&A.nup[r[q]]);
    acc[q] = T(0);
  }
#pragma unroll
  for (int s = 0; s < KMAX; ++s) {
    if (s < klg) {
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        const size_t e = (size_t)s * A.n + r[q];
        if (s < kl[q]) acc[q] = acc[q] + __ldg(&A.aoff[e]) * ldm(&w[__ldg(&A.col[e])]);
      }
    }
  }
#pragma unroll
  for (int t = 0; t < KMAX; ++t) {
    if (t < kug) {
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        const size_t e = (size_t)(A.KL + t) * A.n + r[q];
        if (t < ku[q]) acc[q] = acc[q] + __ldg(&A.aoff[e]) * ldm(&w[__ldg(&A.col[e])]);
      }
    }
  }
}
// diag_r w_r - sum_{all} a_rj w_j
template <typename T, int NR>
__device__ __forceinline__ void spmv_rows(const PersistArgs<T>& A, T (&y)[NR], const T* w, const int (&r)[NR],
                                          int klg, int kug) {
  T acc[NR], dg[NR], wr[NR];
#pragma unroll
  for (int q = 0; q < NR; ++q) {
    dg[q] = __ldg(&A.diag[r[q]]);
    wr[q] = ldm(&w[r[q]]);
  }
  offdiag_sum(A, acc, w, r, klg, kug);
#pragma unroll
  for (int q = 0; q < NR; ++q) y[q] = dg[q] * wr[q] - acc[q];
}

// Preconditioner application z = (LU)^-1 y with the right-hand side formed per
// row by mode (as k_fwd): 0 p-update, 1 x/r-update.  One phase per group of
// the forward sweep, then one per group of the backward sweep.  With spmv0,
// the backward phase of group 0 also forms the following SpMV for its rows
// (MODE 0: u = A z and u.r0 into dots[0]; MODE 1: v = A z, v.r and v.v into
// dots[0..1]): those rows couple only to later groups, whose z is final, and
// the gathered neighbour values serve both sums.  Group-0 rows have no lower
// couplings, so ILU(0) leaves them as they are in A (both k_ilu0 and
// k_ilu0_relax): u_rk = -aoff and u_rr = diag, and that phase reads aoff and
// diag only (w + aoff z rounds exactly as w - luoff z, and 1/diag is the
// stored invd).
template <typename T, int MODE>
__device__ __forceinline__ void pc_apply(const PersistArgs<T>& A, PhaseState& ph, const int* s_lo, const int* s_pre,
                                         double omg_d, double alf_d, double gam_d, bool pending,
                                         double (&dots)[5]) {
  constexpr int NR = NRT<T>;
  const T omg = (T)omg_d, alf = (T)alf_d, gam = (T)gam_d;
  const int G = A.G;
  // The last group normally has no upper couplings (no two rows of a group
  // are coupled and every later row is in a later group); its backward step
  // then needs no other row and is done in the forward pass.
  const bool fuse = A.relax || (A.gku_last == 0);
  // forward phases: one per group, or (relax) group 0 then groups 1..G-1
  // together with their backward step (their upper couplings are dropped)
  const int nfwd = A.relax ? 2 : G;
  for (int ph_i = 0; ph_i < nfwd && ph.ok; ++ph_i) {
    const int ga = ph_i, gb = (A.relax && ph_i == 1) ? G - 1 : ph_i;
    if (tile_count(A, s_pre, ga, gb) > 0) wait_neighbours(A, ph);
    const int klg = ga == gb ? __ldg(&A.gkl[ga]) : A.klB;
    const bool last = fuse && (gb == G - 1 || (A.relax && ga >= 1));
    const int cmax = (A.relax && ga >= 1) ? A.g1 : 0x7fffffff;
    for_rows_g<NR>(A, s_lo, s_pre, ga, gb, [&](const int (&r)[NR], const bool (&ok)[NR]) {
      T y[NR], xo[NR], zo[NR], iv[NR], rn[NR], r0v[NR];
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        if (MODE == 0) {
          if (pending) {  // the previous iteration's x += alf z, r -= alf v (own row)
            zo[q] = ldm(&A.z[r[q]]);
            xo[q] = ldm(&A.x[r[q]]);
            rn[q] = ldm(&A.r[r[q]]) - alf * ldm(&A.v[r[q]]);
          } else {
            rn[q] = ldm(&A.r[r[q]]);
          }
          y[q] = rn[q] + omg * (ldm(&A.p[r[q]]) - alf * ldm(&A.u[r[q]]));
        } else {
          y[q] = ldm(&A.r[r[q]]) - gam * ldm(&A.u[r[q]]);
          xo[q] = ldm(&A.x[r[q]]);
          zo[q] = ldm(&A.z[r[q]]);
          if (A.fuse_upd) r0v[q] = ldm(&A.r0[r[q]]);
        }
        iv[q] = last ? __ldg(&A.invd[r[q]]) : T(1);
      }
      T w[NR];
#pragma unroll
      for (int q = 0; q < NR; ++q) w[q] = y[q];
      lower_sub(A, w, A.z, r, klg, cmax);
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        if (!ok[q]) continue;
        if (MODE == 0) {
          if (pending) {
            A.x[r[q]] = xo[q] + alf * zo[q];
            A.r[r[q]] = rn[q];
          }
          A.p[r[q]] = y[q];
        } else {
          A.x[r[q]] = xo[q] + gam * zo[q];
          A.r[r[q]] = y[q];
          if (A.fuse_upd) {  // r1.r0 and r1.r1 for the identities
            dots[3] += (double)y[q] * (double)r0v[q];
            dots[4] += (double)y[q] * (double)y[q];
          }
        }
        A.z[r[q]] = last ? iv[q] * w[q] : w[q];
      }
    });
    end_phase(A, ph);
  }
  for (int g = A.relax ? 0 : (fuse ? G - 2 : G - 1); g >= 0 && ph.ok; --g) {
    const int2 rr = tile_rows(A, g);
    const int kug = __ldg(&A.gku[g]);
    if (rr.y > rr.x) wait_neighbours(A, ph);
    if (g == 0 && A.spmv0) {
      for_rows<NR>(rr.x, rr.y, [&](const int (&r)[NR], const bool (&ok)[NR]) {
        T w[NR], dg[NR], d1[NR], sa[NR], r0v[NR];
        int ku[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          w[q] = ldm(&A.z[r[q]]);
          dg[q] = __ldg(&A.diag[r[q]]);
          d1[q] = MODE == 0 ? ldm(&A.r0[r[q]]) : ldm(&A.r[r[q]]);
          if (MODE == 1 && A.fuse_upd) r0v[q] = ldm(&A.r0[r[q]]);
          ku[q] = __ldg(&A.nup[r[q]]);
          sa[q] = T(0);
        }
#pragma unroll
        for (int t = 0; t < KMAX; ++t) {
          if (t < kug) {
#pragma unroll
            for (int q = 0; q < NR; ++q) {
              const size_t e = (size_t)(A.KL + t) * A.n + r[q];
              if (t < ku[q]) {
                const T zk = ldm(&A.z[__ldg(&A.col[e])]);
                const T a = __ldg(&A.aoff[e]);
                w[q] = w[q] + a * zk;
                sa[q] = sa[q] + a * zk;
              }
            }
          }
        }
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          if (!ok[q]) continue;
          const T zr = (T(1) / dg[q]) * w[q];
          const T y = dg[q] * zr - sa[q];
          A.z[r[q]] = zr;
          if (MODE == 0) {
            A.u[r[q]] = y;
            dots[0] += (double)y * (double)d1[q];
          } else {
            A.v[r[q]] = y;
            dots[0] += (double)y * (double)d1[q];
            dots[1] += (double)y * (double)y;
            if (A.fuse_upd) dots[2] += (double)y * (double)r0v[q];
          }
        }
      });
      end_phase(A, ph);
      continue;
    }
    for_rows<NR>(rr.x, rr.y, [&](const int (&r)[NR], const bool (&ok)[NR]) {
      T w[NR], iv[NR];
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        w[q] = ldm(&A.z[r[q]]);
        iv[q] = __ldg(&A.invd[r[q]]);
      }
      upper_sub(A, w, A.z, r, kug);
#pragma unroll
      for (int q = 0; q < NR; ++q)
        if (ok[q]) A.z[r[q]] = iv[q] * w[q];
    });
    end_phase(A, ph);
  }
}

// The solve run by one block (tile A.tile of the system A describes).
template <typename T>
__device__ __forceinline__ void bicg_body(const PersistArgs<T>& A) {
  constexpr int NR = NRT<T>;
  const int G = A.G;
  PhaseState ph{0u, 0u, true, true};
  // this tile's group ranges (groups beyond GFLAT are read per phase)
  __shared__ int s_lo[GFLAT], s_pre[GFLAT + 1];
  if (G <= GFLAT && threadIdx.x == 0) {
    int acc = 0;
    for (int g = 0; g < G; ++g) {
      const int2 rr = tile_rows(A, g);
      s_lo[g] = rr.x;
      s_pre[g] = acc;
      acc += rr.y - rr.x;
    }
    s_pre[G] = acc;
  }
  __syncthreads();
  // slot bounds of the SpMV phases (rows of groups spmv0..G-1)
  const int klS = A.spmv0 ? A.klB : A.KL, kuS = A.spmv0 ? A.kuB : A.KU;
  // start: r = b - A x + small, r0 = r, p = u = v = 0 (x is only read here,
  // or zeroed row by row)
  double res0 = 1.0, bet = 0.0;
  {
    double s2[2] = {0.0, 0.0};
    {
      const int klg = A.KL, kug = A.KU;
      for_rows_g<NR>(A, s_lo, s_pre, 0, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
        T term[NR], bq[NR], dg[NR], xq[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          bq[q] = __ldg(&A.b[r[q]]);
          dg[q] = A.xzero ? T(0) : __ldg(&A.diag[r[q]]);
          xq[q] = A.xzero ? T(0) : A.x[r[q]];
        }
        if (A.xzero) {
#pragma unroll
          for (int q = 0; q < NR; ++q) term[q] = bq[q];
        } else {
          offdiag_sum(A, term, A.x, r, klg, kug);
#pragma unroll
          for (int q = 0; q < NR; ++q) term[q] = term[q] + bq[q] - dg[q] * xq[q];
        }
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          if (!ok[q]) continue;
          const T rs = term[q] + (T)SMALL;
          if (A.xzero) A.x[r[q]] = T(0);
          A.r[r[q]] = rs; A.r0[r[q]] = rs;
          A.p[r[q]] = T(0); A.u[r[q]] = T(0); A.v[r[q]] = T(0);
          s2[0] += fabs((double)rs);
          s2[1] += (double)rs * (double)rs;
        }
      });
    }
    put_partials<2>(A, s2, 0);
    end_phase(A, ph);
    grid_barrier(A, ph);
    if (ph.ok) {
      get_totals<2>(A, s2, 0);
      res0 = (A.norm == 1) ? s2[0] : sqrt(s2[1]);
      bet = s2[1];
    }
  }
  double alf = 1.0, bet0 = 1.0, gam = 1.0, rel = 1.0;
  int it = 0, converged = 0, nonfinite = 0;
  int buf = 1;
  bool pending = false;  // fuse_upd: an x/r update waits for the next forward phases
  while (ph.ok && it < A.maxit) {
    ++it;
    const double omg = bet * gam / (alf * bet0 + SMALL);
    double dots[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    pc_apply<T, 0>(A, ph, s_lo, s_pre, omg, alf, gam, pending, dots);
    pending = false;
    if (!ph.ok) break;
    // u = A z, u.r0 (rows of later groups)
    {
      double s1[1] = {dots[0]};
      wait_neighbours(A, ph);
      {
        const int klg = klS, kug = kuS;
        for_rows_g<NR>(A, s_lo, s_pre, A.spmv0, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
          T ur[NR], d1[NR];
#pragma unroll
          for (int q = 0; q < NR; ++q) d1[q] = ldm(&A.r0[r[q]]);
          spmv_rows(A, ur, A.z, r, klg, kug);
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            if (!ok[q]) continue;
            A.u[r[q]] = ur[q];
            s1[0] += (double)ur[q] * (double)d1[q];
          }
        });
      }
      put_partials<1>(A, s1, buf);
      end_phase(A, ph);
      grid_barrier(A, ph);
      if (!ph.ok) break;
      get_totals<1>(A, s1, buf);
      buf ^= 1;
      gam = bet / s1[0];
      bet0 = bet;
    }
    for (double& d : dots) d = 0.0;
    pc_apply<T, 1>(A, ph, s_lo, s_pre, omg, alf, gam, false, dots);
    if (!ph.ok) break;
    // v = A z, v.r, v.v (rows of later groups); with fuse_upd also v.r0 and
    // the r1.r0, r1.r1 sums of the forward phases
    {
      double s5[5] = {dots[0], dots[1], dots[2], dots[3], dots[4]};
      wait_neighbours(A, ph);
      {
        const int klg = klS, kug = kuS;
        for_rows_g<NR>(A, s_lo, s_pre, A.spmv0, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
          T vr[NR], d1[NR], r0v[NR];
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            d1[q] = ldm(&A.r[r[q]]);
            if (A.fuse_upd) r0v[q] = ldm(&A.r0[r[q]]);
          }
          spmv_rows(A, vr, A.z, r, klg, kug);
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            if (!ok[q]) continue;
            A.v[r[q]] = vr[q];
            s5[0] += (double)vr[q] * (double)d1[q];
            s5[1] += (double)vr[q] * (double)vr[q];
            if (A.fuse_upd) s5[2] += (double)vr[q] * (double)r0v[q];
          }
        });
      }
      if (A.fuse_upd) put_partials<5>(A, s5, buf);
      else {
        double s2[2] = {s5[0], s5[1]};
        put_partials<2>(A, s2, buf);
      }
      end_phase(A, ph);
      grid_barrier(A, ph);
      if (!ph.ok) break;
      if (A.fuse_upd) get_totals<5>(A, s5, buf);
      else {
        double s2[2];
        get_totals<2>(A, s2, buf);
        s5[0] = s2[0]; s5[1] = s2[1];
      }
      buf ^= 1;
      alf = s5[0] / fmax(s5[1], SMALL);
      if (A.fuse_upd) {
        // r = r1 - alf v:  |r|^2 = |r1|^2 - 2 alf v.r1 + alf^2 v.v,  r.r0 = r1.r0 - alf v.r0
        const double rr = fmax(s5[4] - 2.0 * alf * s5[0] + alf * alf * s5[1], 0.0);
        rel = sqrt(rr) / res0;
        bet = s5[3] - alf * s5[2];
        pending = true;
        if (!isfinite(rel)) { nonfinite = 1; break; }
        if (rel < A.tol) { converged = 1; break; }
        continue;
      }
    }
    // x += alf z; r -= alf v; stopping test; next bet (own rows only)
    {
      const T a = (T)alf;
      double s3[3] = {0.0, 0.0, 0.0};
      {
        for_rows_g<NR>(A, s_lo, s_pre, 0, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
          T xn[NR], rn[NR], r0v[NR];
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            xn[q] = ldm(&A.x[r[q]]) + a * ldm(&A.z[r[q]]);
            rn[q] = ldm(&A.r[r[q]]) - a * ldm(&A.v[r[q]]);
            r0v[q] = ldm(&A.r0[r[q]]);
          }
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            if (!ok[q]) continue;
            A.x[r[q]] = xn[q];
            A.r[r[q]] = rn[q];
            s3[0] += fabs((double)rn[q]);
            s3[1] += (double)rn[q] * (double)rn[q];
            s3[2] += (double)rn[q] * (double)r0v[q];
          }
        });
      }
      put_partials<3>(A, s3, buf);
      end_phase(A, ph);
      grid_barrier(A, ph);
      if (!ph.ok) break;
      get_totals<3>(A, s3, buf);
      buf ^= 1;
      const double res = (A.norm == 1) ? s3[0] : sqrt(s3[1]);
      rel = res / res0;
      bet = s3[2];
      if (!isfinite(rel)) { nonfinite = 1; break; }
      if (rel < A.tol) { converged = 1; break; }
    }
  }
  // fuse_upd: the last iteration's update (own rows; every tile has passed the
  // last grid barrier, nothing else reads these rows afterwards)
  if (pending && ph.ok) {
    const T a = (T)alf;
    for_rows_g<NR>(A, s_lo, s_pre, 0, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
      T xn[NR], rn[NR];
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        xn[q] = ldm(&A.x[r[q]]) + a * ldm(&A.z[r[q]]);
        rn[q] = ldm(&A.r[r[q]]) - a * ldm(&A.v[r[q]]);
      }
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        if (!ok[q]) continue;
        A.x[r[q]] = xn[q];
        A.r[r[q]] = rn[q];
      }
    });
  }
  if (A.tile == 0 && threadIdx.x == 0) {
    A.st->iter = it;
    A.st->s[S_RELRES] = rel;
    A.st->s[S_RES0] = res0;
    A.st->converged = converged;
    A.st->nonfinite = nonfinite;
    A.st->done = 1;
    A.st->s[S_BET] = bet;
  }
}

// One system: block b works on tile b.
template <typename T>
__global__ void __launch_bounds__(TPB, 4) k_bicg_persistent(PersistArgs<T> A) {
  __shared__ PersistArgs<T> sA;
  if (threadIdx.x == 0) {
    sA = A;
    sA.ntiles = gridDim.x;
    sA.tile = blockIdx.x;
  }
  __syncthreads();
  bicg_body<T>(sA);
}

// Several independent systems (an ensemble) in one launch: bmap[b] = (member,
// tile) of block b.  Each member has its own tiles, progress counters,
// partial sums, barrier and device state, so members share nothing but the
// launch and each stops at its own stopping test.
template <typename T>
__global__ void __launch_bounds__(TPB, 4) k_bicg_batched(const PersistArgs<T>* __restrict__ members,
                                                         const int2* __restrict__ bmap) {
  __shared__ PersistArgs<T> sA;
  if (threadIdx.x == 0) {
    const int2 mt = bmap[blockIdx.x];
    sA = members[mt.x];
    sA.tile = mt.y;
  }
  __syncthreads();
  bicg_body<T>(sA);
}

// Failure-detection check of the waits above: one block runs tile 0 of a
// two-tile system whose tile 1 never runs, so tile 1 never publishes a phase
// and never arrives at a grid barrier.  which = 0: the neighbour wait
// (phase 1 of tile 1); 1: the grid barrier (2 arrivals needed).  The wait
// must give up after A.spin_limit polls and set A.bar->err; out[0] = 1 when
// the block saw it fail, out[1] the barrier arrivals it saw.
template <typename T>
__global__ void __launch_bounds__(TPB) k_persist_wait_probe(PersistArgs<T> A, int which, int* out) {
  __shared__ PersistArgs<T> sA;
  if (threadIdx.x == 0) {
    sA = A;
    sA.tile = 0;
    sA.ntiles = 2;
  }
  __syncthreads();
  PhaseState ph{1u, 0u, false, true};
  if (which == 0) wait_neighbours(sA, ph);
  else grid_barrier(sA, ph);
  if (threadIdx.x == 0) {
    out[0] = ph.ok ? 0 : 1;
    out[1] = (int)ld_acquire(&sA.bar->count);
  }
}

// Factor of the two-phase preconditioner: ILU(0) of A without the couplings
// among rows of groups >= 1 (g1 = first such row).  Group-0 rows have no
// lower couplings: u_jj = diag_j and their upper entries are A's.  A row r of
// a later group keeps only its couplings to group 0: l_rj = a_rj / diag_j and
// u_rr = diag_r - sum_j l_rj a_jr; its other entries are zero.  Every row is
// independent, so one launch over all rows suffices.
template <typename T>
__global__ void __launch_bounds__(TPB) k_ilu0_relax(int n, int KL, int g1, const int* __restrict__ col,
                                                    const signed char* __restrict__ nlo,
                                                    const signed char* __restrict__ nup,
                                                    const T* __restrict__ aoff, const T* __restrict__ diag,
                                                    T* __restrict__ luoff, T* __restrict__ invd) {
  for (int r = blockIdx.x * TPB + threadIdx.x; r < n; r += gridDim.x * TPB) {
    const int kl = nlo[r], ku = nup[r];
    if (r < g1) {
      invd[r] = T(1) / diag[r];
      for (int t = 0; t < ku; ++t) luoff[(size_t)(KL + t) * n + r] = -aoff[(size_t)(KL + t) * n + r];
      for (int s = 0; s < kl; ++s) luoff[(size_t)s * n + r] = T(0);
      continue;
    }
    T d = diag[r];
    for (int s = 0; s < kl; ++s) {
      const size_t e = (size_t)s * n + r;
      const int j = col[e];
      T lij = T(0);
      if (j != r && j < g1) {
        lij = -aoff[e] * (T(1) / diag[j]);
        const int nuj = nup[j];
        for (int t2 = 0; t2 < nuj; ++t2) {
          const size_t e2 = (size_t)(KL + t2) * n + j;
          if (col[e2] == r) d = d - lij * (-aoff[e2]);
        }
      }
      luoff[e] = lij;
    }
    for (int t = 0; t < ku; ++t) luoff[(size_t)(KL + t) * n + r] = T(0);
    invd[r] = T(1) / d;
  }
}

}  // namespace cms
