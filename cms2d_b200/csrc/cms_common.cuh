// Shared device helpers: launch geometry, warp/block reductions with a
// deterministic last-block finish, and the device-resident solver scalars.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace cms {

constexpr int TPB = 256;           // threads per block of the row kernels
constexpr int MAXG = 16;           // groups kept in a launch table (more: one merged group)
constexpr int KMAX = 8;            // ELL slots per side handled by the unrolled loops
constexpr double SMALL = 1.0e-15;  // `small`, source/main/definitions.F90:93

// Scalar slots of the device state (doubles).
enum Slot : int {
  S_BET = 0, S_BET0, S_OMG, S_ALF, S_GAM, S_RES, S_RES0, S_UKR0, S_SUM1, S_SUM2,
  S_TOL, S_RELRES, S_RO, S_EPS11, S_RO0, S_SCALE,
  S_SCALE1 = 16,  // GMRES: scale of v_1..v_4 (slots 16..19)
  S_RS1 = 20,     // GMRES: rs1(1..4) at 21..24 (index 20 unused)
  S_C = 25,       // c(1..3) at 26..28
  S_S = 29,       // s(1..3) at 30..32
  S_HH = 33,      // hh(j,i), j=1..4, i=1..3 at 33 + (j-1)*3 + (i-1)  (33..44)
  S_Y = 45,       // y(1..3) at 46..48
  S_NRM2 = 49,    // sums handed back to the host
  S_NRM2B = 50,
  S_RMOM = 51,
  S_TRUE0 = 52,
  S_TRUE1 = 53,
  S_IRSCALE = 54, // refinement: norm of the residual handed to the FP32 solve
  S_NSLOTS = 64
};

// Grid barrier of the persistent solver kernel (cms_persist.cuh).
struct GridBar {
  unsigned int count;  // blocks arrived at the current barrier
  unsigned int gen;    // barrier generation
  int err;             // 1: a block gave up waiting (bounded spin)
  int pad;
};

struct DevState {
  double s[S_NSLOTS];
  int done;       // 1: the solve has stopped (converged or capped)
  int iter;       // BiCGStab iterations / GMRES cycles executed
  int maxit;      // cap
  int norm;       // 1 = L1, 2 = L2
  int active;     // GMRES: Arnoldi of the current cycle still running
  int ifinal;     // GMRES: Arnoldi steps of the current cycle
  int stop;       // GMRES: converged in the current cycle
  int inner;      // GMRES: Arnoldi steps in total
  int converged;  // 1 when the stopping test passed
  int nonfinite;  // 1 when a non-finite value reached a reduction
  GridBar bar;
  int pad[2];
  unsigned int ticket[8];
};

// Per-launch group table: rows [start[g], start[g+1]) use kl[g] lower and
// ku[g] upper slots; blocks [blk[g], blk[g+1]) cover group g.
struct GroupTab {
  int ng;
  int start[MAXG + 1];
  int blk[MAXG + 1];
  int kl[MAXG];
  int ku[MAXG];
};

__device__ __forceinline__ int tab_group(const GroupTab& t, int b) {
  int g = 0;
#pragma unroll 1
  for (int q = 1; q < t.ng; ++q)
    if (b >= t.blk[q]) g = q;
  return g;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sums of NS values; the result is valid in thread 0.
template <int NS>
__device__ __forceinline__ void block_sum(double (&v)[NS]) {
  __shared__ double sm[NS][TPB / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NS; ++q) v[q] = warp_sum(v[q]);
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NS; ++q) sm[q][wid] = v[q];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      double t = (lane < (int)(blockDim.x >> 5)) ? sm[q][lane] : 0.0;
      v[q] = warp_sum(t);
    }
  }
  __syncthreads();
}

// Reduces NS per-thread values over the whole grid.  Block partials land in
// partials[q * gridDim.x + blockIdx.x]; the last block to finish sums them in
// a fixed order (deterministic) and returns true in its thread 0 with the
// totals in v.  ticket is reset for the next use.
template <int NS>
__device__ __forceinline__ bool grid_sum(double (&v)[NS], double* partials, unsigned int* ticket) {
  __shared__ bool last;
  block_sum<NS>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NS; ++q) partials[(size_t)q * gridDim.x + blockIdx.x] = v[q];
    __threadfence();
    unsigned int t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double acc[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    acc[q] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) acc[q] += __ldcg(&partials[(size_t)q * gridDim.x + b]);
  }
  block_sum<NS>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NS; ++q) v[q] = acc[q];
    *ticket = 0u;
    return true;
  }
  return false;
}

template <typename T> __device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// Polls of a device-side wait before it gives up and reports an error.
constexpr unsigned int kSpinLimit = 1u << 22;

// gpu-scope acquire load / release store of a progress flag
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// relaxed load of a flag; a fence_acquire after the last one orders the loads that follow
__device__ __forceinline__ unsigned int ld_relaxed(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acquire() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

}  // namespace cms
