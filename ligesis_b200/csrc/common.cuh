// Shared host/device plumbing for the LigeSIS B200 prover library: status codes, CUDA error
// propagation, and the twiddle table every transform reads.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "gl64.cuh"

namespace lgs {

// Largest transform size supported: twiddle table holds g_TW^e for e < 2^TW_LOG.
constexpr unsigned TW_LOG = 22;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct ShapeError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct OracleError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct DeviceTimeout : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define LGS_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::lgs::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " +  \
                             __FILE__ + ":" + std::to_string(__LINE__));                    \
  } while (0)
// Every kernel launch of the library is followed by this check, which also counts it.
#define LGS_LAUNCH_CHECK()                \
  do {                                    \
    LGS_CUDA(cudaGetLastError());         \
    ::lgs::count_launch();                \
  } while (0)

// Process-wide count of kernels this library has launched (lgs_launch_count()).
void count_launch();
uint64_t thread_launches();      // launches counted by the calling host thread
void adjust_launches(int64_t n);  // graph replays add their kernels; captures remove theirs

inline unsigned ilog2(uint64_t x) {
  unsigned k = 0;
  while ((uint64_t(1) << k) < x) ++k;
  return k;
}
inline unsigned cdiv(uint64_t a, uint64_t b) { return (unsigned)((a + b - 1) / b); }

// Device-side view of the twiddle table: tw[e] = g^e for the order-2^TW_LOG generator g.
// The order-2^k root raised to e is tw[e << (TW_LOG - k)].
struct Twiddles {
  const u64* tw = nullptr;
};

}  // namespace lgs
