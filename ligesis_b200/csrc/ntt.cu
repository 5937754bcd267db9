// Batched Goldilocks DFTs in natural order: out[j] = sum_k in[k] g^(jk), g = the order-N
// two-adic generator.  This is the transform the reference takes from p3-dft's
// `Radix2Dit::dft` for its Reed-Solomon encodings (pcs/src/ligesis.rs:222-235, rate 1/2: the
// input is a length-n vector zero-padded to N = 2n) and for Basefold's interleaved codewords
// (pcs/src/basefold.rs:341-382).  EF ("dft_algebra") vectors are transformed coordinate-wise.
//
// Sizes up to 2^12 run as one shared-memory transform per CTA.  Larger sizes use the four-step
// split N = N1 * N2: pass A does length-N1 column transforms (stride N2) and multiplies by
// g_N^(j1*k2); pass B does length-N2 row transforms and writes X[j1 + N1*j2].  Zero-padded
// inputs are never read.
#include "kernels.cuh"

namespace lgs {

__device__ __forceinline__ unsigned brev(unsigned x, unsigned bits) {
  return bits ? (__brev(x) >> (32 - bits)) : 0;
}

// In-place radix-2 DIT over `cnt` transforms of length 2^logL held in shared memory in
// bit-reversed order: element e of transform t lives at s[t*ts + e*es].  Output natural order.
__device__ void smem_dit(u64* s, unsigned logL, unsigned cnt, unsigned ts, unsigned es,
                         const u64* __restrict__ tw) {
  const unsigned L = 1u << logL, halfL = L >> 1;
  const unsigned total = cnt * halfL;
  for (unsigned st = 1; st <= logL; ++st) {
    const unsigned half = 1u << (st - 1);
    const unsigned tshift = TW_LOG - st;
    for (unsigned idx = threadIdx.x; idx < total; idx += blockDim.x) {
      unsigned t = idx >> (logL - 1);
      unsigned bf = idx & (halfL - 1);
      unsigned k = bf & (half - 1);
      unsigned i0 = ((bf >> (st - 1)) << st) + k;
      unsigned a_off = t * ts + i0 * es, b_off = a_off + half * es;
      u64 a = s[a_off];
      u64 b = s[b_off];
      if (k) b = gl_mul(b, __ldg(tw + ((u64)k << tshift)));
      s[a_off] = gl_add(a, b);
      s[b_off] = gl_sub(a, b);
    }
    __syncthreads();
  }
}

// Whole transform in shared memory: one CTA handles `per_cta` vectors of length N = 2^logN.
__global__ void ntt_small_kernel(const u64* __restrict__ in, size_t in_stride, size_t n_in,
                                 u64* __restrict__ out, size_t out_stride, unsigned logN,
                                 unsigned per_cta, size_t batch, const u64* __restrict__ tw) {
  extern __shared__ u64 sm[];
  const unsigned N = 1u << logN;
  const size_t b0 = (size_t)blockIdx.x * per_cta;
  const unsigned cnt = (unsigned)min((size_t)per_cta, batch - b0);
  for (unsigned idx = threadIdx.x; idx < cnt * N; idx += blockDim.x) {
    unsigned t = idx >> logN, e = idx & (N - 1);
    u64 v = e < n_in ? in[(b0 + t) * in_stride + e] : 0;
    sm[t * N + brev(e, logN)] = v;
  }
  __syncthreads();
  smem_dit(sm, logN, cnt, N, 1, tw);
  for (unsigned idx = threadIdx.x; idx < cnt * N; idx += blockDim.x) {
    unsigned t = idx >> logN, e = idx & (N - 1);
    out[(b0 + t) * out_stride + e] = sm[t * N + e];
  }
}

// Pass A: CTA = TC consecutive columns k2 of one vector; transform along k1 (length N1).
__global__ void ntt_passA_kernel(const u64* __restrict__ in, size_t in_stride, size_t n_in,
                                 u64* __restrict__ y, unsigned logN, unsigned logN1,
                                 unsigned logTC, const u64* __restrict__ tw) {
  extern __shared__ u64 sm[];
  const unsigned N1 = 1u << logN1, logN2 = logN - logN1, N2 = 1u << logN2, TC = 1u << logTC;
  const size_t b = blockIdx.y;
  const unsigned k2_0 = blockIdx.x << logTC;
  const u64* src = in + b * in_stride;
  for (unsigned idx = threadIdx.x; idx < (N1 << logTC); idx += blockDim.x) {
    unsigned k1 = idx >> logTC, c = idx & (TC - 1);
    size_t e = ((size_t)k1 << logN2) + k2_0 + c;
    u64 v = e < n_in ? src[e] : 0;
    sm[(brev(k1, logN1) << logTC) + c] = v;
  }
  __syncthreads();
  smem_dit(sm, logN1, TC, 1, TC, tw);
  u64* dst = y + b * ((size_t)1 << logN);
  const unsigned tshift = TW_LOG - logN;
  for (unsigned idx = threadIdx.x; idx < (N1 << logTC); idx += blockDim.x) {
    unsigned j1 = idx >> logTC, c = idx & (TC - 1);
    unsigned k2 = k2_0 + c;
    u64 v = sm[idx];
    unsigned ex = (unsigned)(((u64)j1 * k2) & (((u64)1 << logN) - 1));
    if (ex) v = gl_mul(v, __ldg(tw + ((u64)ex << tshift)));
    dst[((size_t)j1 << logN2) + k2] = v;
  }
  (void)N2;
}

// Pass B: CTA = TR consecutive rows j1; transform along k2 (length N2, contiguous);
// write X[j1 + N1 * j2].
__global__ void ntt_passB_kernel(const u64* __restrict__ y, u64* __restrict__ out,
                                 size_t out_stride, unsigned logN, unsigned logN1,
                                 unsigned logTR, const u64* __restrict__ tw) {
  extern __shared__ u64 sm[];
  const unsigned logN2 = logN - logN1, N2 = 1u << logN2, TR = 1u << logTR;
  const unsigned pitch = N2 + 1;
  const size_t b = blockIdx.y;
  const unsigned j1_0 = blockIdx.x << logTR;
  const u64* src = y + b * ((size_t)1 << logN) + ((size_t)j1_0 << logN2);
  for (unsigned idx = threadIdx.x; idx < (TR << logN2); idx += blockDim.x) {
    unsigned r = idx >> logN2, k2 = idx & (N2 - 1);
    sm[r * pitch + brev(k2, logN2)] = src[idx];
  }
  __syncthreads();
  smem_dit(sm, logN2, TR, pitch, 1, tw);
  u64* dst = out + b * out_stride;
  for (unsigned idx = threadIdx.x; idx < (TR << logN2); idx += blockDim.x) {
    unsigned r = idx & (TR - 1), j2 = idx >> logTR;
    dst[j1_0 + r + ((size_t)j2 << logN1)] = sm[r * pitch + j2];
  }
}

__global__ void twiddle_kernel(u64* tw, u64 g, unsigned logn) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >> logn) return;
  tw[i] = gl_pow(g, i);
}

void build_twiddles(u64* d_tw, cudaStream_t st) {
  u64 g = gl_two_adic_generator(TW_LOG);
  size_t n = (size_t)1 << TW_LOG;
  twiddle_kernel<<<cdiv(n, 256), 256, 0, st>>>(d_tw, g, TW_LOG);
  LGS_LAUNCH_CHECK();
}

void ntt_batch(const u64* in, size_t in_stride, size_t n_in, u64* out, size_t out_stride,
               unsigned logN, size_t batch, u64* scratch, const u64* tw, cudaStream_t st) {
  if (logN > TW_LOG) throw ShapeError("transform larger than the twiddle table");
  if (batch == 0) return;
  const size_t N = (size_t)1 << logN;
  if (n_in > N) n_in = N;
  if (logN <= 12) {
    unsigned per_cta = logN >= 10 ? 1 : (1u << (10 - logN));
    size_t smem = (size_t)per_cta * N * 8;
    unsigned grid = cdiv(batch, per_cta);
    ntt_small_kernel<<<grid, 256, smem, st>>>(in, in_stride, n_in, out, out_stride, logN,
                                              per_cta, batch, tw);
    LGS_LAUNCH_CHECK();
    return;
  }
  if (!scratch) throw std::runtime_error("ntt_batch: scratch required above 2^12");
  unsigned logN1 = (logN + 1) / 2, logN2 = logN - logN1;
  unsigned logTC = logN1 >= 12 ? 0 : std::min(12 - logN1, logN2);
  unsigned logTR = logN2 >= 12 ? 0 : std::min(12 - logN2, logN1);
  if (logTR > 5) logTR = 5;
  size_t smA = ((size_t)1 << (logN1 + logTC)) * 8;
  size_t smB = ((size_t)(((size_t)1 << logN2) + 1) << logTR) * 8;  // both <= 33 KB
  dim3 gA((unsigned)(((size_t)1 << logN2) >> logTC), (unsigned)batch);
  ntt_passA_kernel<<<gA, 256, smA, st>>>(in, in_stride, n_in, scratch, logN, logN1, logTC, tw);
  LGS_LAUNCH_CHECK();
  dim3 gB((unsigned)(((size_t)1 << logN1) >> logTR), (unsigned)batch);
  ntt_passB_kernel<<<gB, 256, smB, st>>>(scratch, out, out_stride, logN, logN1, logTR, tw);
  LGS_LAUNCH_CHECK();
}

// out[c][r] = in[r][c] for a rows x cols matrix of u64, `batch` matrices back to back.
__global__ void transpose_kernel(const u64* __restrict__ in, u64* __restrict__ out, size_t rows,
                                 size_t cols) {
  __shared__ u64 tile[32][33];
  const size_t bz = blockIdx.z;
  in += bz * rows * cols;
  out += bz * rows * cols;
  size_t c0 = (size_t)blockIdx.x * 32, r0 = (size_t)blockIdx.y * 32;
  for (unsigned i = threadIdx.y; i < 32; i += blockDim.y) {
    size_t r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[i][threadIdx.x] = in[r * cols + c];
  }
  __syncthreads();
  for (unsigned i = threadIdx.y; i < 32; i += blockDim.y) {
    size_t c = c0 + i, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][i];
  }
}

void transpose_u64(const u64* in, u64* out, size_t rows, size_t cols, size_t batch,
                   cudaStream_t st) {
  if (!rows || !cols || !batch) return;
  dim3 grid(cdiv(cols, 32), cdiv(rows, 32), (unsigned)batch);
  transpose_kernel<<<grid, dim3(32, 8), 0, st>>>(in, out, rows, cols);
  LGS_LAUNCH_CHECK();
}

}  // namespace lgs
