// FP32 inner BiCGStab of iterative refinement in reduced form.
//
// On a multicolour ordering group 0 is an independent set placed first: its
// rows couple only to rows of the later groups (set B).  With
// A = [D0 A0B; AB0 ABB] the ILU(0) preconditioner of a two-group split is
// M = (D~ + L) D~^-1 (D~ + U) with D~ = diag(D0, S), S the diagonal of the
// Schur complement C = ABB - AB0 D0^-1 A0B, and a short calculation gives
//
//   (I + L D~^-1)^-1 A (D~ + U)^-1 = diag(I, C S^-1),
//
// so right-preconditioned BiCGStab on A M^-1 runs on an operator similar to
// diag(I, C S^-1): the group-0 block is the identity.  This file solves the
// reduced system instead, C S^-1 y = b_B - AB0 D0^-1 b_0 on the B rows with
// x_B = S^-1 y and x_0 = D0^-1 (b_0 - A0B x_B): half the unknowns, one
// unit-diagonal gather per operator application and no triangular sweep.
// Couplings among B rows (telescoping interfaces) stay in C exactly.  The
// reduced residual equals the full system's residual on B, and the FP64
// residual of the refinement makes the answer independent of the inner
// operator's rounding.
//
// Storage.  C S^-1 = I - Chat: Chat's off-diagonals in ELL slot-major order
// over the reduced rows i = r - g1 (ccol: device column, coff: value, ccnt:
// count per row), built per solve by k_schur_diag and k_schur_off from the
// FP32 matrix; sinv[r] = 1/d_r for group-0 rows and 1/s_r (s_r = C_rr) for B
// rows.  Vectors are indexed by device row (the B rows of the refinement's
// FP32 work arrays).
//
// The persistent kernels.  One block per tile (the tiles of the persistent
// ILU(0) kernel: tile t's B rows are toff[g][t]..toff[g][t+1] for g >= 1).
// Two iteration forms: the single-reduction form (schur_body_sr, the
// default layouts; one grid barrier per iteration, described at its
// definition) and the three-phase form (schur_body), a BiCGStab iteration
// in three phases:
//   P0  the previous iteration's y/r update and the new search direction p
//       (own rows, no neighbour values);
//   A   nu = Chat p (after the neighbour tiles have finished P0) and r0.nu,
//       reduced at a grid barrier;
//   B   t = Chat s with s = r - alpha nu formed on the fly for each gathered
//       neighbour, and t.s, t.t, r0.t, s.s, r0.s, reduced at a grid barrier;
// the next residual norm comes from ||r||^2 = s.s - 2 w t.s + w^2 t.t and the
// next r0.r from r0.s - w r0.t.  Waits and barriers are those of the
// persistent ILU(0) kernel (bounded, cms_persist.cuh).
//
// Measured on the three-phase form, one B200, same box, 1M-cell inlet flow
// step (timesteps/s): 5.50 as written; couplings packed as one 8-byte
// (column, value) element and (r, nu) interleaved for one 8-byte gather,
// 5.24-5.33; P0 and its neighbour wait dropped by forming each gathered
// neighbour's new direction from a 16-byte (r, nu, p, t) gather in
// alternating buffers, 4.72; the tile's columns and counts cached in shared
// memory for the launch, 5.10.  Separate 4-byte streams keep more loads in
// flight per thread.
#pragma once
#include "cms_persist.cuh"

namespace cms {

constexpr int KSC = 16;  // largest off-diagonal count of a reduced row the kernels take
constexpr double kDiverge = 100.0;  // single-reduction form: stop when the residual is this many times the best
constexpr int kStall = 100;         // single-reduction form: stop after this many iterations without a new best

struct SchurArgs {
  int n, g1, nB, KL, G;
  int KC;                  // slots of Chat (largest count)
  int ntiles, tile;
  const int* toff;         // [G][ntiles+1] tile row ranges per group
  const int* dep_ptr;      // neighbour tiles under Chat's couplings
  const int* dep_idx;
  unsigned int* progress;  // [ntiles * kProgressStride] (zero at launch)
  const int* ccol;         // [KC][nB]
  const float* coff;       // [KC][nB]
  const signed char* ccnt; // [nB]
  const int* col;          // A's ELL (device order)
  const signed char* nlo;
  const signed char* nup;
  const float* aoff;
  const float* sinv;       // [n]
  const float* b;
  float* x;
  float *r, *r0, *p, *nu, *t, *y;
  // single-reduction form only: the transpose slot map (ctr[e] = offset of
  // Chat's entry (k, i) for the entry e = (i, k)), u = op r, q = op nu, f0,
  // and s, t interleaved per row (one 8-byte gather in X)
  const int* ctr;          // [KC][nB]
  float *u, *q, *f0;
  float2* s_t;
  float* yb;               // the iterate with the smallest residual so far
  double* part;            // [2][NSMAX][ntiles]
  GridBar* bar;
  DevState* st;
  int maxit;
  double tol;
  unsigned int spin_limit;
};

// sinv: 1/d_r for group-0 rows, 1/s_r for B rows with
// s_r = d_r - sum_{j in group 0} a_rj a_jr / d_j (A's off-diagonals are
// -aoff; products accumulated in FP64).
__global__ void __launch_bounds__(TPB) k_schur_diag(int n, int g1, int KL, const int* __restrict__ col,
                                                    const signed char* __restrict__ nlo,
                                                    const signed char* __restrict__ nup,
                                                    const float* __restrict__ aoff, const float* __restrict__ diag,
                                                    float* __restrict__ sinv) {
  for (int r = blockIdx.x * TPB + threadIdx.x; r < n; r += gridDim.x * TPB) {
    const float dr = diag[r];
    if (r < g1) {
      sinv[r] = 1.0f / dr;
      continue;
    }
    double c = dr;
    const int kl = nlo[r];
    for (int s = 0; s < kl; ++s) {
      const size_t e = (size_t)s * n + r;
      const int j = col[e];
      if (j >= g1) continue;
      const int nuj = nup[j];
      for (int t2 = 0; t2 < nuj; ++t2) {
        const size_t e2 = (size_t)(KL + t2) * n + j;
        if (col[e2] == r) c -= (double)aoff[e] * (double)aoff[e2] / (double)diag[j];
      }
    }
    sinv[r] = (float)(1.0 / c);
  }
}

// Chat's off-diagonals of reduced row i (r = g1 + i):
// coff_rk = (aoff_rk [k in B] + sum_{j in group 0} aoff_rj aoff_jk / d_j) / s_k.
// A thread's columns and FP64 accumulators live in shared memory, so four
// blocks fit on an SM (with them in registers the kernel took 110 registers
// and two blocks; its chains of dependent gathers need the extra warps).
__global__ void __launch_bounds__(TPB, 4) k_schur_off(int n, int g1, int nB, int KL, int KC,
                                                   const int* __restrict__ col, const signed char* __restrict__ nlo,
                                                   const signed char* __restrict__ nup,
                                                   const float* __restrict__ aoff, const float* __restrict__ diag,
                                                   const float* __restrict__ sinv, const int* __restrict__ ccol,
                                                   const signed char* __restrict__ ccnt, float* __restrict__ coff) {
  __shared__ double s_acc[KSC][TPB];  // this thread's columns and accumulators: column threadIdx.x
  __shared__ int s_cc[KSC][TPB];
  double* acc = &s_acc[0][threadIdx.x];
  int* cc = &s_cc[0][threadIdx.x];
  for (int i = blockIdx.x * TPB + threadIdx.x; i < nB; i += gridDim.x * TPB) {
    const int r = g1 + i;
    const int kc = ccnt[i];
    for (int q = 0; q < kc; ++q) {
      cc[q * TPB] = ccol[(size_t)q * nB + i];
      acc[q * TPB] = 0.0;
    }
    auto add = [&](int k, double v) {  // a row's columns are distinct
      for (int q = 0; q < kc; ++q)
        if (cc[q * TPB] == k) {
          acc[q * TPB] += v;
          break;
        }
    };
    const int kl = nlo[r], ku = nup[r];
    for (int s = 0; s < kl + ku; ++s) {
      const size_t e = (size_t)(s < kl ? s : KL + (s - kl)) * n + r;
      const int k = col[e];
      const double a = aoff[e];
      if (k >= g1) {
        add(k, a);
        continue;
      }
      const double w = a / (double)diag[k];  // k is a group-0 row j
      const int nuj = nup[k];
      for (int t2 = 0; t2 < nuj; ++t2) {
        const size_t e2 = (size_t)(KL + t2) * n + k;
        const int k2 = col[e2];
        if (k2 != r) add(k2, w * (double)aoff[e2]);
      }
    }
    for (int q = 0; q < KC; ++q)
      coff[(size_t)q * nB + i] = q < kc ? (float)(acc[q * TPB] * (double)sinv[cc[q * TPB]]) : 0.0f;
  }
}

// This block's partial sums of NS values into buffer buf: warp sums in
// shared memory, then warp q adds value q over the block's warps (fixed
// order) and its lane 0 stores it.  The stores are ordered before the
// phase's progress release by end_phase's __syncthreads.
template <int NS, int BS>
__device__ __forceinline__ void put_partials_bs(const SchurArgs& A, double (&v)[NS], int buf) {
  constexpr int NW = BS / 32;
  __shared__ double sm[NS][NW];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NS; ++q) v[q] = warp_sum(v[q]);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NS; ++q) sm[q][wid] = v[q];
  }
  __syncthreads();
  for (int q = wid; q < NS; q += NW) {
    const double x = warp_sum(lane < NW ? sm[q][lane] : 0.0);
    if (lane == 0) A.part[((size_t)buf * NSMAX + q) * A.ntiles + A.tile] = x;
  }
}

// After a grid barrier: the grid totals, value q summed by warp q (lane l
// adds tiles l, l + 32, ... in that order, then a butterfly), so every block
// forms the same bits; then shared with the block.  A lane's loads for up
// to 256 tiles are issued before their adds (one round trip; the missing ones
// add 0, which changes no bits).
template <int NS, int BS>
__device__ __forceinline__ void get_totals_w0(const SchurArgs& A, double (&tot)[NS], int buf) {
  constexpr int NW = BS / 32;
  __shared__ double bc[NS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nt = A.ntiles;
  for (int q = wid; q < NS; q += NW) {
    const double* src = A.part + ((size_t)buf * NSMAX + q) * nt;
    double acc = 0.0;
    for (int b = lane; b < nt; b += 256) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = b + 32 * u < nt ? __ldcg(src + b + 32 * u) : 0.0;
#pragma unroll
      for (int u = 0; u < 8; ++u) acc += v[u];
    }
    acc = warp_sum(acc);
    if (lane == 0) bc[q] = acc;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NS; ++q) tot[q] = bc[q];
}

// Rows of this tile in groups ga..gb as one index space (ranges in shared
// memory: s_lo first row of each group's range, s_pre prefix counts).
template <int NR, typename F>
__device__ __forceinline__ void for_tile_rows(const int* s_lo, const int* s_pre, int ga, int gb, F&& f) {
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

// acc[q] - sum_s coff[s] * w(col) over the reduced row's KC slots, w(k)
// given by a functor of the gathered column.  Every slot is read, the padding
// ones too (column = the row itself, coefficient 0): the loads then wait on
// no count, one dependent step less per batch (measured faster than reading
// only the row's count of slots, although it loads ~30 % more coefficients
// on the telescoping inlet).
template <int NR, typename W>
__device__ __forceinline__ void chat_sub(const SchurArgs& A, float (&acc)[NR], const int (&r)[NR], W&& w) {
#pragma unroll
  for (int s = 0; s < KSC; ++s) {
    if (s < A.KC) {
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        const size_t e = (size_t)s * A.nB + (r[q] - A.g1);
        acc[q] = acc[q] - __ldg(&A.coff[e]) * w(__ldg(&A.ccol[e]));
      }
    }
  }
}

template <int BS, int NR>
__device__ __forceinline__ void schur_body(const SchurArgs& A) {
  const int G = A.G;
  PhaseState ph{0u, 0u, true, true};
  __shared__ int s_lo[GFLAT], s_pre[GFLAT + 1];
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int g = 0; g < G; ++g) {
      const int* o = A.toff + (size_t)g * (A.ntiles + 1) + A.tile;
      s_lo[g] = __ldg(o);
      s_pre[g] = acc;
      acc += __ldg(o + 1) - __ldg(o);
    }
    s_pre[G] = acc;
  }
  __syncthreads();
  const int n = A.n, g1 = A.g1;
  // start: r = r0 = b_B - AB0 D0^-1 b_0, p = nu = t = y = 0
  double res0 = 0.0, rho = 0.0;
  {
    double s1[1] = {0.0};
    for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
      float acc[NR];
      int kl[NR];
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        acc[q] = __ldg(&A.b[r[q]]);
        kl[q] = __ldg(&A.nlo[r[q]]);
      }
#pragma unroll
      for (int s = 0; s < KMAX; ++s) {
        if (s < A.KL) {
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            if (s < kl[q]) {
              const size_t e = (size_t)s * n + r[q];
              const int j = __ldg(&A.col[e]);
              if (j < g1) acc[q] = acc[q] + __ldg(&A.aoff[e]) * (__ldg(&A.b[j]) * __ldg(&A.sinv[j]));
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        if (!ok[q]) continue;
        A.r[r[q]] = acc[q]; A.r0[r[q]] = acc[q];
        A.p[r[q]] = 0.0f; A.nu[r[q]] = 0.0f; A.t[r[q]] = 0.0f; A.y[r[q]] = 0.0f;
        s1[0] += (double)acc[q] * (double)acc[q];
      }
    });
    put_partials_bs<1, BS>(A, s1, 0);
    end_phase(A, ph);
    grid_barrier(A, ph);
    if (ph.ok) {
      get_totals_w0<1, BS>(A, s1, 0);
      res0 = sqrt(s1[0]);
      rho = s1[0];
    }
  }
  double alf = 1.0, omg = 1.0, bet = 0.0, rel = res0 > 0.0 ? 1.0 : 0.0;
  int it = 0, converged = res0 > 0.0 ? 0 : 1, nonfinite = 0, buf = 1;
  bool pending = false;  // an iteration's y/r update not yet applied
  while (ph.ok && !converged && it < A.maxit) {
    ++it;
    // P0: the pending update, then p = r + bet (p - omg nu)
    {
      const float a = (float)alf, w = (float)omg, be = (float)bet;
      for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
        float rr[NR], pv[NR], nv[NR], tv[NR], yv[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          rr[q] = ldm(&A.r[r[q]]);
          pv[q] = ldm(&A.p[r[q]]);
          nv[q] = ldm(&A.nu[r[q]]);
          if (pending) {
            tv[q] = ldm(&A.t[r[q]]);
            yv[q] = ldm(&A.y[r[q]]);
          }
        }
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          if (!ok[q]) continue;
          float rn = rr[q];
          if (pending) {
            const float sv = rr[q] - a * nv[q];
            A.y[r[q]] = yv[q] + a * pv[q] + w * sv;
            rn = sv - w * tv[q];
            A.r[r[q]] = rn;
          }
          A.p[r[q]] = rn + be * (pv[q] - w * nv[q]);
        }
      });
      pending = false;
      end_phase(A, ph);
    }
    // A: nu = Chat p, r0.nu
    {
      double s1[1] = {0.0};
      wait_neighbours(A, ph);
      for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
        float acc[NR], r0v[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          acc[q] = ldm(&A.p[r[q]]);
          r0v[q] = ldm(&A.r0[r[q]]);
        }
        chat_sub(A, acc, r, [&](int k) { return ldm(&A.p[k]); });
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          if (!ok[q]) continue;
          A.nu[r[q]] = acc[q];
          s1[0] += (double)r0v[q] * (double)acc[q];
        }
      });
      put_partials_bs<1, BS>(A, s1, buf);
      end_phase(A, ph);
      grid_barrier(A, ph);
      if (!ph.ok) break;
      get_totals_w0<1, BS>(A, s1, buf);
      buf ^= 1;
      // a breakdown (r0.nu = 0) ends this inner solve with the iterate so far
      // (the refinement's FP64 residual takes over); a non-finite sum is an error
      if (!isfinite(s1[0])) { nonfinite = 1; break; }
      if (s1[0] == 0.0) break;
      alf = rho / s1[0];
    }
    // B: t = Chat s, s = r - alf nu; t.s, t.t, r0.t, s.s, r0.s
    {
      double s5[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      const float a = (float)alf;
      for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
        float acc[NR], sv[NR], r0v[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          sv[q] = ldm(&A.r[r[q]]) - a * ldm(&A.nu[r[q]]);
          r0v[q] = ldm(&A.r0[r[q]]);
          acc[q] = sv[q];
        }
        chat_sub(A, acc, r, [&](int k) { return ldm(&A.r[k]) - a * ldm(&A.nu[k]); });
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          if (!ok[q]) continue;
          A.t[r[q]] = acc[q];
          const double tq = acc[q], sq = sv[q], oq = r0v[q];
          s5[0] += tq * sq;
          s5[1] += tq * tq;
          s5[2] += oq * tq;
          s5[3] += sq * sq;
          s5[4] += oq * sq;
        }
      });
      put_partials_bs<5, BS>(A, s5, buf);
      end_phase(A, ph);
      grid_barrier(A, ph);
      if (!ph.ok) break;
      get_totals_w0<5, BS>(A, s5, buf);
      buf ^= 1;
      omg = s5[0] / fmax(s5[1], SMALL);
      const double rr = fmax(s5[3] - 2.0 * omg * s5[0] + omg * omg * s5[1], 0.0);
      const double rho1 = s5[4] - omg * s5[2];
      rel = sqrt(rr) / res0;
      if (!isfinite(rel) || !isfinite(omg) || !isfinite(rho1)) { nonfinite = 1; break; }
      pending = true;  // y += alf p + omg s is valid even at a breakdown below
      if (rel < A.tol) { converged = 1; continue; }
      // breakdown of the next step (omg = 0 or r0.r = 0): stop with this iterate
      if (omg == 0.0 || rho1 == 0.0) break;
      bet = (rho1 / rho) * (alf / omg);
      rho = rho1;
    }
  }
  // the last update (y only), x_B = S^-1 y, then x_0 = D0^-1 (b_0 + sum aoff x_B)
  if (ph.ok && !nonfinite) {
    const float a = (float)alf, w = (float)omg;
    for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
      float yv[NR], si[NR];
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        yv[q] = ldm(&A.y[r[q]]);
        if (pending) yv[q] = yv[q] + a * ldm(&A.p[r[q]]) + w * (ldm(&A.r[r[q]]) - a * ldm(&A.nu[r[q]]));
        si[q] = __ldg(&A.sinv[r[q]]);
      }
#pragma unroll
      for (int q = 0; q < NR; ++q)
        if (ok[q]) A.x[r[q]] = yv[q] * si[q];
    });
    end_phase(A, ph);
    grid_barrier(A, ph);
    if (ph.ok) {
      for_tile_rows<NR>(s_lo, s_pre, 0, 0, [&](const int (&r)[NR], const bool (&ok)[NR]) {
        float acc[NR], si[NR];
        int ku[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          acc[q] = __ldg(&A.b[r[q]]);
          si[q] = __ldg(&A.sinv[r[q]]);
          ku[q] = __ldg(&A.nup[r[q]]);
        }
#pragma unroll
        for (int t2 = 0; t2 < KMAX; ++t2) {
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            if (t2 < ku[q]) {
              const size_t e = (size_t)(A.KL + t2) * n + r[q];
              acc[q] = acc[q] + __ldg(&A.aoff[e]) * ldm(&A.x[__ldg(&A.col[e])]);
            }
          }
        }
#pragma unroll
        for (int q = 0; q < NR; ++q)
          if (ok[q]) A.x[r[q]] = acc[q] * si[q];
      });
    }
  }
  if (A.tile == 0 && threadIdx.x == 0) {
    A.st->iter = it;
    A.st->s[S_RELRES] = rel;
    A.st->s[S_RES0] = res0;
    A.st->converged = converged;
    A.st->nonfinite = nonfinite;
    A.st->done = 1;
  }
}

// Single-reduction form of the same iteration (the reorganisation of L. T.
// Yang and R. P. Brent, "The improved BiCGStab method for large and sparse
// unsymmetric linear systems on parallel distributed memory architectures",
// 2002): one grid barrier per iteration instead of two.  With op = I - Chat,
// u = op r and q = op nu (nu = op p), the search direction's image and t
// follow without a product of their own,
//   nu' = u' + bet (nu - omg q),   t = op s = u - alf q,
// and r0.nu', which alf needs before q is known, from
//   r0.nu' = r0.u' + bet (r0.nu - omg r0.q),   r0.u' = f0.r',   f0 = op^T r0
// (f0 once per launch; Chat's pattern is structurally symmetric, so op^T's
// row i gathers over row i's own columns with the coefficients at the
// transpose slots ctr).  An iteration is two phases:
//   X  r = s - omg t (own rows and each gathered neighbour), u = op r, the
//      pending y update, p = r + bet (p - omg nu), nu = u + bet (nu - omg q);
//   Y  (after the neighbour tiles have finished X) q = op nu, s = r - alf nu,
//      t = u - alf q, and t.s, t.t, s.s, r0.s, r0.t, f0.s, f0.t, r0.q, r0.nu,
//      reduced at a grid barrier.
// r0.nu is summed from the vector (not carried by the recurrence), so the
// recurrence extrapolates one iteration at a time.  The result is the
// iterate with the smallest residual (kept in yb when it is not the last),
// and a residual kDiverge times the smallest ends the solve: on the 1M-cell
// inlet's pressure-correction systems a long FP32 solve can pass 1e-3 and
// drift to 1e-2; the refinement then restarts from the best iterate's
// residual (measured: median/90th/largest final residuals of those solves
// 3.3e-4/1.4e-2/6.9e-2 against 4.4e-4/2.1e-2/0.19 returning the last iterate,
// same step time; stopping at 10 times the best was 3 % slower).  kStall
// iterations without a smaller residual end it too: an FP32 solve asked for
// more than its arithmetic can reach would otherwise spend the whole budget
// of an outer solve (a 1e-9 solve's 600 iterations) on one restart.  Y overwrites s and t of
// its own rows: every neighbour that gathers them in X has finished X (the
// neighbour wait), and the next X starts after the grid barrier.
template <int BS, int NR>
__device__ __forceinline__ void schur_body_sr(const SchurArgs& A) {
  const int G = A.G;
  PhaseState ph{0u, 0u, true, true};
  __shared__ int s_lo[GFLAT], s_pre[GFLAT + 1];
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int g = 0; g < G; ++g) {
      const int* o = A.toff + (size_t)g * (A.ntiles + 1) + A.tile;
      s_lo[g] = __ldg(o);
      s_pre[g] = acc;
      acc += __ldg(o + 1) - __ldg(o);
    }
    s_pre[G] = acc;
  }
  __syncthreads();
  const int n = A.n, g1 = A.g1;
  // start, first phase: r0 = s = b_B - AB0 D0^-1 b_0, y = 0
  for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
    float acc[NR];
    int kl[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) {
      acc[q] = __ldg(&A.b[r[q]]);
      kl[q] = __ldg(&A.nlo[r[q]]);
    }
#pragma unroll
    for (int s = 0; s < KMAX; ++s) {
      if (s < A.KL) {
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          if (s < kl[q]) {
            const size_t e = (size_t)s * n + r[q];
            const int j = __ldg(&A.col[e]);
            if (j < g1) acc[q] = acc[q] + __ldg(&A.aoff[e]) * (__ldg(&A.b[j]) * __ldg(&A.sinv[j]));
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < NR; ++q) {
      if (!ok[q]) continue;
      A.r0[r[q]] = acc[q]; A.s_t[r[q]] = make_float2(acc[q], 0.0f); A.y[r[q]] = 0.0f; A.yb[r[q]] = 0.0f;
    }
  });
  end_phase(A, ph);
  // start, second phase: f0 = op^T r0, u = nu = op r0, p = r0; r0.r0, f0.r0
  double res0 = 0.0, rho = 0.0, alf = 0.0;
  int converged = 0, nonfinite = 0;
  bool stop = false;
  {
    double s2[2] = {0.0, 0.0};
    wait_neighbours(A, ph);
    for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
      float ua[NR], fa[NR], r0v[NR];
      int kc[NR];
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        r0v[q] = ldm(&A.r0[r[q]]);
        ua[q] = r0v[q];
        fa[q] = r0v[q];
        kc[q] = __ldg(&A.ccnt[r[q] - g1]);
      }
#pragma unroll
      for (int s = 0; s < KSC; ++s) {
        if (s < A.KC) {
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            if (s < kc[q]) {
              const size_t e = (size_t)s * A.nB + (r[q] - g1);
              const float rk = ldm(&A.r0[__ldg(&A.ccol[e])]);
              ua[q] = ua[q] - __ldg(&A.coff[e]) * rk;
              fa[q] = fa[q] - __ldg(&A.coff[__ldg(&A.ctr[e])]) * rk;
            }
          }
        }
      }
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        if (!ok[q]) continue;
        A.f0[r[q]] = fa[q]; A.u[r[q]] = ua[q]; A.nu[r[q]] = ua[q]; A.p[r[q]] = r0v[q];
        s2[0] += (double)r0v[q] * (double)r0v[q];
        s2[1] += (double)fa[q] * (double)r0v[q];
      }
    });
    put_partials_bs<2, BS>(A, s2, 0);
    end_phase(A, ph);
    grid_barrier(A, ph);
    if (ph.ok) {
      get_totals_w0<2, BS>(A, s2, 0);
      res0 = sqrt(s2[0]);
      rho = s2[0];
      if (res0 == 0.0) converged = 1;
      else if (!isfinite(s2[1]) || !isfinite(res0)) nonfinite = 1;
      else if (s2[1] == 0.0) stop = true;  // breakdown before the first step
      else alf = rho / s2[1];
    }
  }
  double omg = 0.0, bet = 0.0, alf_n = alf, rel = res0 > 0.0 ? 1.0 : 0.0;
  // squared residual norms: the tests below need no square root or division
  const double tol2 = (A.tol * res0) * (A.tol * res0);
  double rr_last = res0 * res0, best2 = rr_last;
  int it_best = 0;
  int it = 0, buf = 1;
  bool pending = false;  // an iteration's y update not yet applied
  bool save = false;     // the pending iterate has the smallest residual so far (yb holds the best otherwise)
  while (ph.ok && !converged && !nonfinite && !stop && it < A.maxit) {
    ++it;
    // X: r = s - omg t, u = op r, the pending y update (kept in yb too when
    // it is the best iterate so far), p and nu
    if (it > 1) {
      const float a = (float)alf, w = (float)omg, be = (float)bet;
      const bool keep = save;
      for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
        float sv[NR], yv[NR], pv[NR], nv[NR], qv[NR], rv[NR], acc[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          const float2 st2 = ldm(&A.s_t[r[q]]);
          sv[q] = st2.x;
          rv[q] = st2.x - w * st2.y;
          yv[q] = ldm(&A.y[r[q]]);
          pv[q] = ldm(&A.p[r[q]]);
          nv[q] = ldm(&A.nu[r[q]]);
          qv[q] = ldm(&A.q[r[q]]);
          acc[q] = rv[q];
        }
        chat_sub(A, acc, r, [&](int k) {
          const float2 st2 = ldm(&A.s_t[k]);
          return st2.x - w * st2.y;
        });
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          if (!ok[q]) continue;
          const float yn = yv[q] + a * pv[q] + w * sv[q];
          A.y[r[q]] = yn;
          if (keep) A.yb[r[q]] = yn;
          A.u[r[q]] = acc[q];
          A.p[r[q]] = rv[q] + be * (pv[q] - w * nv[q]);
          A.nu[r[q]] = acc[q] + be * (nv[q] - w * qv[q]);
        }
      });
      pending = false;
      alf = alf_n;
      end_phase(A, ph);
    }
    // Y: q = op nu, s = r - alf nu, t = u - alf q, nine sums
    {
      double s9[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      const float a = (float)alf, w = (float)omg;
      const bool first = it == 1;
      wait_neighbours(A, ph);
      for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
        float rv[NR], nv[NR], uv[NR], r0v[NR], f0v[NR], acc[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          r0v[q] = ldm(&A.r0[r[q]]);
          const float2 st2 = ldm(&A.s_t[r[q]]);
          rv[q] = first ? r0v[q] : st2.x - w * st2.y;
          nv[q] = ldm(&A.nu[r[q]]);
          uv[q] = ldm(&A.u[r[q]]);
          f0v[q] = ldm(&A.f0[r[q]]);
          acc[q] = nv[q];
        }
        chat_sub(A, acc, r, [&](int k) { return ldm(&A.nu[k]); });
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          if (!ok[q]) continue;
          const float sn = rv[q] - a * nv[q], tn = uv[q] - a * acc[q];
          A.q[r[q]] = acc[q];
          A.s_t[r[q]] = make_float2(sn, tn);
          const double sd = sn, td = tn, od = r0v[q], fd = f0v[q];
          s9[0] += td * sd;
          s9[1] += td * td;
          s9[2] += sd * sd;
          s9[3] += od * sd;
          s9[4] += od * td;
          s9[5] += fd * sd;
          s9[6] += fd * td;
          s9[7] += od * (double)acc[q];
          s9[8] += od * (double)nv[q];
        }
      });
      put_partials_bs<9, BS>(A, s9, buf);
      grid_barrier(A, ph);  // (no progress release: every tile skips the same one)
      if (!ph.ok) break;
      get_totals_w0<9, BS>(A, s9, buf);
      buf ^= 1;
      omg = s9[0] / fmax(s9[1], SMALL);
      const double rr = fmax(s9[2] - 2.0 * omg * s9[0] + omg * omg * s9[1], 0.0);
      const double rho1 = s9[3] - omg * s9[4];
      rr_last = rr;
      if (!isfinite(rr) || !isfinite(omg) || !isfinite(rho1)) { rel = rr; nonfinite = 1; break; }
      pending = true;  // y += alf p + omg s is valid even at a breakdown below
      save = rr < best2;
      if (save) {
        best2 = rr;
        it_best = it;
      }
      if (rr < tol2) { converged = 1; continue; }
      // breakdown of the next step (omg = 0, r0.r = 0 or r0.nu = 0): stop with this iterate
      if (omg == 0.0 || rho1 == 0.0) break;
      // divergence: the residual kDiverge times the best one; the best iterate
      // is the result (the refinement restarts from its residual)
      if (rr > (kDiverge * kDiverge) * best2) break;
      // stagnation: kStall iterations without a smaller residual
      if (it - it_best >= kStall) break;
      bet = (rho1 / rho) * (alf / omg);
      rho = rho1;
      const double tau = (s9[5] - omg * s9[6]) + bet * (s9[8] - omg * s9[7]);
      if (!isfinite(tau) || !isfinite(bet)) { nonfinite = 1; break; }
      if (tau == 0.0) break;
      alf_n = rho / tau;
    }
  }
  // the best iterate: the last one (its y update still pending) or yb;
  // x_B = S^-1 y, then x_0 = D0^-1 (b_0 + sum aoff x_B)
  const bool last = !pending || save;
  if (!nonfinite && it > 0) rel = sqrt(last ? rr_last : best2) / res0;
  if (ph.ok && !nonfinite) {
    const float a = (float)alf, w = (float)omg;
    for_tile_rows<NR>(s_lo, s_pre, 1, G - 1, [&](const int (&r)[NR], const bool (&ok)[NR]) {
      float yv[NR], si[NR];
#pragma unroll
      for (int q = 0; q < NR; ++q) {
        if (last) {
          yv[q] = ldm(&A.y[r[q]]);
          if (pending) yv[q] = yv[q] + a * ldm(&A.p[r[q]]) + w * ldm(&A.s_t[r[q]]).x;
        } else {
          yv[q] = ldm(&A.yb[r[q]]);
        }
        si[q] = __ldg(&A.sinv[r[q]]);
      }
#pragma unroll
      for (int q = 0; q < NR; ++q)
        if (ok[q]) A.x[r[q]] = yv[q] * si[q];
    });
    end_phase(A, ph);
    grid_barrier(A, ph);
    if (ph.ok) {
      for_tile_rows<NR>(s_lo, s_pre, 0, 0, [&](const int (&r)[NR], const bool (&ok)[NR]) {
        float acc[NR], si[NR];
        int ku[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) {
          acc[q] = __ldg(&A.b[r[q]]);
          si[q] = __ldg(&A.sinv[r[q]]);
          ku[q] = __ldg(&A.nup[r[q]]);
        }
#pragma unroll
        for (int t2 = 0; t2 < KMAX; ++t2) {
#pragma unroll
          for (int q = 0; q < NR; ++q) {
            if (t2 < ku[q]) {
              const size_t e = (size_t)(A.KL + t2) * n + r[q];
              acc[q] = acc[q] + __ldg(&A.aoff[e]) * ldm(&A.x[__ldg(&A.col[e])]);
            }
          }
        }
#pragma unroll
        for (int q = 0; q < NR; ++q)
          if (ok[q]) A.x[r[q]] = acc[q] * si[q];
      });
    }
  }
  if (A.tile == 0 && threadIdx.x == 0) {
    A.st->iter = it;
    A.st->s[S_RELRES] = rel;
    A.st->s[S_RES0] = res0;
    A.st->converged = converged;
    A.st->nonfinite = nonfinite;
    A.st->done = 1;
  }
}

// Block and row layouts of the reduced kernel: threads per block, rows per
// thread per batch, and the iteration form (0: three phases and two grid
// barriers per iteration, schur_body; 1: single reduction, schur_body_sr).
// cms_solver_opts.reduced_layout picks one by its position (1-based).
#define CMS_SCHUR_LAYOUTS(X) X(256, 2, 0) X(512, 2, 0) X(512, 4, 0) X(1024, 2, 0) X(1024, 2, 1) X(512, 2, 1) \
  X(256, 2, 1)
constexpr int kSchurLayouts = 7;

template <int BS, int NR, int SR>
__device__ __forceinline__ void schur_run(const SchurArgs& A) {
  if constexpr (SR != 0) schur_body_sr<BS, NR>(A);
  else schur_body<BS, NR>(A);
}

// Several independent systems (an ensemble) in one launch: bmap[b] = (member,
// tile) of block b; members share nothing but the launch.
template <int BS, int NR, int SR>
__global__ void __launch_bounds__(BS, 1024 / BS) k_schur_batched(const SchurArgs* __restrict__ members,
                                                                  const int2* __restrict__ bmap) {
  __shared__ SchurArgs sA;
  if (threadIdx.x == 0) {
    const int2 mt = bmap[blockIdx.x];
    sA = members[mt.x];
    sA.tile = mt.y;
  }
  __syncthreads();
  schur_run<BS, NR, SR>(sA);
}

// One system: block b works on tile b.
template <int BS, int NR, int SR>
__global__ void __launch_bounds__(BS, 1024 / BS) k_schur_bicg(SchurArgs A) {
  __shared__ SchurArgs sA;
  if (threadIdx.x == 0) {
    sA = A;
    sA.ntiles = gridDim.x;
    sA.tile = blockIdx.x;
  }
  __syncthreads();
  schur_run<BS, NR, SR>(sA);
}

// Kernels, block size and form of layout k.
struct SchurLayout {
  const void* single;
  const void* batched;
  int bs;
  int sr;
};
inline SchurLayout schur_layout(int k) {
  int q = 0;
#define CMS_SCHUR_PICK(B, R, F)                                                                            \
  if (q++ == k)                                                                                            \
    return SchurLayout{(const void*)k_schur_bicg<B, R, F>, (const void*)k_schur_batched<B, R, F>, B, F};
  CMS_SCHUR_LAYOUTS(CMS_SCHUR_PICK)
#undef CMS_SCHUR_PICK
  return SchurLayout{(const void*)k_schur_bicg<256, 2, 0>, (const void*)k_schur_batched<256, 2, 0>, 256, 0};
}

}  // namespace cms
