// Allocation-free residual check of the solve() boundary.
//
// Some hosts may not allocate device memory at the point where they need the
// normalised residual of a momentum or pressure-correction system: a caller
// that runs under a fixed device-memory budget handed out by its own pool, a
// caller that must not trigger an implicit device synchronisation (cudaMalloc
// and cudaFree may synchronise the device), or a host model that only checks
// convergence and never builds a solver handle.  For them this file offers one
// entry point that uses no cudaMalloc, no cudaFree and no allocating library
// routine: its only scratch is the file-scope device array below, reserved
// when the library is loaded and held by every GPU that loads it until exit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "cms_common.cuh"
#include "cmsgpu.h"

namespace {

constexpr int kMaxBlocks = CMS_NOALLOC_MAX_CELLS / cms::TPB;  // one partial sum per block
// [0, kMaxBlocks): block partial sums; kMaxBlocks: the result; the next 8 bytes: the ticket
constexpr int kScratchDoubles = kMaxBlocks + 2;
static_assert(CMS_NOALLOC_MAX_CELLS % cms::TPB == 0, "max cells must be a multiple of the block size");

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Message of the last failed call of this thread.
thread_local char g_err[256] = "";

// ap = (sum_k acoef - sp)/relax; ss += (1-relax)*phi*ap;
// res = iwet*(sum_k acoef*phi_nb + ss - ap*phi)/ap; rmom = sqrt(sum res^2 / ncells)
__global__ void __launch_bounds__(cms::TPB) k_residual_noalloc(int n, int nmf, const int* __restrict__ c2c,
                                                                const int* __restrict__ ncface,
                                                                const int* __restrict__ iwet,
                                                                const double* __restrict__ acoef, double* ss,
                                                                const double* __restrict__ sp, double* res,
                                                                const double* __restrict__ phi, double relax,
                                                                double* scratch) {
  const int i = blockIdx.x * cms::TPB + threadIdx.x;
  double v[1] = {0.0};
  if (i < n) {
    const double rinv = 1.0 / relax, relaxm = 1.0 - relax;
    const int nf = ncface[i];
    const double phii = phi[i];
    double sa = 0.0, sn = 0.0;
    for (int k = 0; k < nf; ++k) {
      const double a = acoef[(size_t)i * nmf + k];
      sa = sa + a;
      sn = sn + a * phi[c2c[(size_t)i * nmf + k] - 1];
    }
    const double ap = (sa - sp[i]) * rinv;
    const double ssi = ss[i] + relaxm * phii * ap;
    ss[i] = ssi;
    const double ri = double(iwet[i]) * (sn + ssi - ap * phii) / ap;
    res[i] = ri;
    v[0] = ri * ri;
  }
  unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + kMaxBlocks + 1);
  if (cms::grid_sum<1>(v, scratch, ticket)) scratch[kMaxBlocks] = sqrt(v[0] / (double)n);
}

// Resolves the device address of the scratch array in the current device's
// context.  Done on every call: it allocates nothing and costs a lookup, and a
// cached address would go stale after cudaDeviceReset (the module is loaded
// again in the new context).
double* scratch_for_current_device(int* rc) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    std::snprintf(g_err, sizeof(g_err), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    *rc = CMS_DEVICE_ERROR;
    return nullptr;
  }
  *rc = CMS_OK;
  return static_cast<double*>(p);
}

int device_error(const char* what, cudaError_t e) {
  std::snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
  return CMS_DEVICE_ERROR;
}

}  // namespace

extern "C" int cms_solve_residual_noalloc_d(int ncells, int ncellsD, int nmaxfaces, const int* cell2cell,
                                            const int* ncface, const int* iwet, const double* acoef, double* ss,
                                            const double* sp, double* res, const double* phi, double relax,
                                            double* rmom, void* stream) {
  if (ncells <= 0 || ncellsD < ncells || nmaxfaces <= 0 || !cell2cell || !ncface || !iwet || !acoef || !ss || !sp ||
      !res || !phi || !rmom || relax == 0.0) {
    std::snprintf(g_err, sizeof(g_err), "bad argument");
    return CMS_BAD_ARGUMENT;
  }
  if (ncells > CMS_NOALLOC_MAX_CELLS) {
    std::snprintf(g_err, sizeof(g_err), "ncells = %d exceeds the allocation-free limit of %d cells", ncells,
                  CMS_NOALLOC_MAX_CELLS);
    return CMS_BAD_ARGUMENT;
  }
  int rc = CMS_OK;
  double* scratch = scratch_for_current_device(&rc);
  if (!scratch) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the ticket must start at zero; the partials are overwritten by every block
  cudaError_t e = cudaMemsetAsync(scratch + kMaxBlocks + 1, 0, sizeof(double), s);
  if (e != cudaSuccess) return device_error("cudaMemsetAsync", e);
  const int nb = (ncells + cms::TPB - 1) / cms::TPB;
  k_residual_noalloc<<<nb, cms::TPB, 0, s>>>(ncells, nmaxfaces, cell2cell, ncface, iwet, acoef, ss, sp, res, phi,
                                             relax, scratch);
  if ((e = cudaGetLastError()) != cudaSuccess) return device_error("kernel launch", e);
  if ((e = cudaMemcpyAsync(rmom, scratch + kMaxBlocks, sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return device_error("cudaMemcpyAsync", e);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return device_error("cudaStreamSynchronize", e);
  if (!std::isfinite(*rmom)) {
    std::snprintf(g_err, sizeof(g_err), "rmom is not finite");
    return CMS_NONFINITE;
  }
  g_err[0] = '\0';
  return CMS_OK;
}

extern "C" const char* cms_noalloc_last_error(void) { return g_err; }
