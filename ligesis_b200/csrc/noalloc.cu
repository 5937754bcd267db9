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
// a host-side stand-in for the array's name, so its device address is looked up once per device
// with cudaGetSymbolAddress, on that device's first call; make that first call before any stream
// capture.  Every call shares the array and it keeps the last call's contents: the copies of the
// factors are rewritten and every partial sum a call reads is written by that same call first,
// so nothing needs clearing.  Calls that overlap on the GPU (other streams, other host threads)
// race on the array.
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

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mu;
ef2* g_na_addr[NA_MAX_DEVICES] = {};

// Device address of the scratch on the current device (looked up on its first use there).
ef2* scratch_address(int dev) {
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw CudaError(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_na_addr[dev] = (ef2*)p;
  }
  return g_na_addr[dev];
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
    LGS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES)
      return set_error(LGS_ERR_BAD_ARG, "lgs_sumcheck_prove_noalloc: device index too large");
    ef2* scratch = scratch_address(dev);
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
