// lgs_sumcheck_prove_noalloc: the product sumcheck prover for callers that must not allocate
// device memory.
//
// Who needs it: a host process whose device memory is owned by another allocator (a framework's
// caching allocator that has already reserved most of HBM, where a foreign cudaMalloc fails or
// fragments its pool), and latency-critical serving loops where cudaMalloc / cudaFree would
// stall on device-wide synchronisation.  Such callers hand in device buffers for the inputs and
// outputs; the working storage comes from a fixed array in this file instead of an allocation.
//
// The scratch is a file-scope __device__ array of NA_ELEMS F_{p^2} values (3 x 2^16 + 16 x 296 x
// 4 = 215,552 values of 16 bytes, about 3.3 MiB) that every GPU loading the library holds until
// the process exits.  It holds the working copies of the d
// factors (the sumcheck folds them in place) and the per-round partial sums.  Host code only has
// a host-side stand-in for the array's name, so its device address is looked up with
// cudaGetSymbolAddress on the first call in each CUDA context (normally a device's primary
// context) and cached for that context; make that first call before any stream capture.
// Every call shares the array and it keeps the last call's contents: the copies of the
// factors are rewritten and every partial sum a call reads is written by that same call first,
// so nothing needs clearing.  Calls that overlap on the GPU (other streams, other host threads)
// race on the array.
#include <cuda.h>
#include <mutex>
#include <string>

#include "../../include/lgs.h"
#include "kernels.cuh"

namespace lgs {
namespace {

constexpr unsigned NA_MAX_K = 16;  // at most 2^16 evaluations per factor
constexpr unsigned NA_MAX_D = 3;   // at most 3 factors
constexpr size_t NA_POLY_ELEMS = (size_t)NA_MAX_D << NA_MAX_K;
constexpr size_t NA_PART_ELEMS = (size_t)NA_MAX_K * SC_MAX_BLOCKS * (NA_MAX_D + 1);
constexpr size_t NA_ELEMS = NA_POLY_ELEMS + NA_PART_ELEMS;

__device__ __align__(256) ef2 g_noalloc_scratch[NA_ELEMS];

// The address of a __device__ symbol belongs to a CUDA context, not to a device index: after
// cudaDeviceReset, or under a driver-API context the caller made current, a device's old
// address is not mapped.  So the cache is keyed on the current context.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
constexpr int NA_MAX_CONTEXTS = 64;
std::mutex g_na_mu;
CUcontext g_na_ctx[NA_MAX_CONTEXTS] = {};
ef2* g_na_addr[NA_MAX_CONTEXTS] = {};
int g_na_used = 0;

CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess || !p || q != cudaDriverEntryPointSuccess)
      throw CudaError("cuCtxGetCurrent is not available from the driver");
    fn = (CtxGetCurrentFn)p;
  }
  return fn;
}

// Device address of the scratch in the current context (looked up on its first use there).
ef2* scratch_address() {
  std::lock_guard<std::mutex> lk(g_na_mu);
  CUcontext ctx = nullptr;
  if (ctx_get_current()(&ctx) != CUDA_SUCCESS || !ctx)
    throw CudaError("lgs_sumcheck_prove_noalloc: no current CUDA context");
  for (int i = 0; i < g_na_used; ++i)
    if (g_na_ctx[i] == ctx) return g_na_addr[i];
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    throw CudaError(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
  // A full table (64 contexts seen) drops its oldest entry; that context is likely gone.
  if (g_na_used == NA_MAX_CONTEXTS) {
    for (int i = 1; i < NA_MAX_CONTEXTS; ++i) {
      g_na_ctx[i - 1] = g_na_ctx[i];
      g_na_addr[i - 1] = g_na_addr[i];
    }
    --g_na_used;
  }
  int slot = g_na_used++;
  g_na_ctx[slot] = ctx;
  g_na_addr[slot] = (ef2*)p;
  return (ef2*)p;
}

}  // namespace

lgs_status set_error(lgs_status s, const std::string& msg);  // capi.cu
}  // namespace lgs

extern "C" lgs_status lgs_sumcheck_prove_noalloc(const uint64_t* polys_dev, unsigned d,
                                                 unsigned k, const uint64_t* challenges_dev,
                                                 uint64_t* rounds_out_dev,
                                                 uint64_t* finals_out_dev, void* stream) {
  using namespace lgs;
  try {
    if (!polys_dev || !challenges_dev || !rounds_out_dev || !finals_out_dev)
      return set_error(LGS_ERR_BAD_ARG, "lgs_sumcheck_prove_noalloc: null pointer");
    if (d < 1 || d > NA_MAX_D || k < 1 || k > NA_MAX_K)
      return set_error(LGS_ERR_BAD_SHAPE,
                           "lgs_sumcheck_prove_noalloc: needs 1 <= d <= 3 factors and "
                           "1 <= k <= 16 variables (its fixed scratch holds 3 x 2^16 values)");
    if (sumcheck_partials_elems(k, d) > NA_PART_ELEMS)
      return set_error(LGS_ERR_INTERNAL, "lgs_sumcheck_prove_noalloc: partials exceed scratch");
    int dev = 0;
    LGS_CUDA(cudaGetDevice(&dev));  // makes the device's primary context current if none is
    ef2* scratch = scratch_address();
    cudaStream_t st = (cudaStream_t)stream;
    const size_t len = (size_t)1 << k;
    ef2* polys[NA_MAX_D];
    for (unsigned j = 0; j < d; ++j) {
      polys[j] = scratch + j * len;
      LGS_CUDA(cudaMemcpyAsync(polys[j], polys_dev + 2 * j * len, len * sizeof(ef2),
                               cudaMemcpyDeviceToDevice, st));
    }
    sumcheck_prove_dev(polys, d, k, (const ef2*)challenges_dev, (ef2*)rounds_out_dev,
                       (ef2*)finals_out_dev, scratch + NA_POLY_ELEMS, st);
    return LGS_OK;
  } catch (const std::exception& e) {
    return set_error(LGS_ERR_CUDA, e.what());
  }
}
