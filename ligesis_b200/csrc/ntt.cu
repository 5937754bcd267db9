// Batched Goldilocks DFTs in natural order: out[j] = sum_k in[k] g^(jk), g = the order-N
// two-adic generator.  This is the transform the reference takes from p3-dft's
// `Radix2Dit::dft` for its Reed-Solomon encodings (pcs/src/ligesis.rs:222-235, rate 1/2: the
// input is a length-n vector zero-padded to N = 2n) and for Basefold's interleaved codewords
// (pcs/src/basefold.rs:341-382).  EF ("dft_algebra") vectors are transformed coordinate-wise.
//
// Sizes up to 2^12 run as one shared-memory transform per CTA.  Larger sizes use the four-step
// split N = N1 * N2 with radix-8 Stockham column transforms (lanes walk adjacent columns, so
// every global access is coalesced): pass A transforms the length-N1 columns k2 and writes
// Z[k2][j1] * g_N^(j1*k2) (transposed), pass B transforms the length-N2 columns j1 of Z and
// writes X[j1 + N1*j2].  Zero-padded inputs are never read.
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
    u64 v = e < n_in ? gl_canon(in[(b0 + t) * in_stride + e]) : 0;
    sm[t * N + brev(e, logN)] = v;
  }
  __syncthreads();
  smem_dit(sm, logN, cnt, N, 1, tw);
  for (unsigned idx = threadIdx.x; idx < cnt * N; idx += blockDim.x) {
    unsigned t = idx >> logN, e = idx & (N - 1);
    out[(b0 + t) * out_stride + e] = sm[t * N + e];
  }
}

// ---- radix-8/4/2 Stockham column transforms ------------------------------------------------
// Small in-register DFTs v'[q] = sum_r v[r] w_R^(rq) (natural order in and out), radix-2 DIT on
// the bit-reversed registers.  The order-8 root is 2^120, so every twiddle inside them is a
// shift (w_4 = 2^48, w_8^3 = 2^168).
template <int R>
__device__ __forceinline__ void dft_small(u64* v);
template <>
__device__ __forceinline__ void dft_small<2>(u64* v) {
  u64 t = v[0];
  v[0] = gl_add(t, v[1]);
  v[1] = gl_sub(t, v[1]);
}
template <>
__device__ __forceinline__ void dft_small<4>(u64* v) {
  u64 b0 = gl_add(v[0], v[2]), b1 = gl_sub(v[0], v[2]);
  u64 b2 = gl_add(v[1], v[3]), b3 = gl_sub(v[1], v[3]);
  u64 t = gl_mul_pow2(b3, 48);
  v[0] = gl_add(b0, b2);
  v[2] = gl_sub(b0, b2);
  v[1] = gl_add(b1, t);
  v[3] = gl_sub(b1, t);
}
template <>
__device__ __forceinline__ void dft_small<8>(u64* v) {
  // bit-reversed order a = v[0,4,2,6,1,5,3,7]
  u64 a0 = gl_add(v[0], v[4]), a1 = gl_sub(v[0], v[4]);
  u64 a2 = gl_add(v[2], v[6]), a3 = gl_sub(v[2], v[6]);
  u64 a4 = gl_add(v[1], v[5]), a5 = gl_sub(v[1], v[5]);
  u64 a6 = gl_add(v[3], v[7]), a7 = gl_sub(v[3], v[7]);
  a3 = gl_mul_pow2(a3, 48);
  a7 = gl_mul_pow2(a7, 48);
  u64 b0 = gl_add(a0, a2), b2 = gl_sub(a0, a2), b1 = gl_add(a1, a3), b3 = gl_sub(a1, a3);
  u64 b4 = gl_add(a4, a6), b6 = gl_sub(a4, a6), b5 = gl_add(a5, a7), b7 = gl_sub(a5, a7);
  b5 = gl_mul_pow2(b5, GL_LOG2_OMEGA8);
  b6 = gl_mul_pow2(b6, (2 * GL_LOG2_OMEGA8) % 192);
  b7 = gl_mul_pow2(b7, (3 * GL_LOG2_OMEGA8) % 192);
  v[0] = gl_add(b0, b4);
  v[4] = gl_sub(b0, b4);
  v[1] = gl_add(b1, b5);
  v[5] = gl_sub(b1, b5);
  v[2] = gl_add(b2, b6);
  v[6] = gl_sub(b2, b6);
  v[3] = gl_add(b3, b7);
  v[7] = gl_sub(b3, b7);
}

template <int LOGL>
struct ColCfg {
  static constexpr int L = 1 << LOGL;
  static constexpr int C = (4096 >> LOGL) < 1 ? 1 : ((4096 >> LOGL) > 16 ? 16 : (4096 >> LOGL));
  static constexpr int T = (C * L / 8) < 32 ? 32 : (C * L / 8);
  static constexpr int R0 = LOGL >= 3 ? 8 : (LOGL == 2 ? 4 : 2);
  static constexpr size_t SMEM = (size_t)L * (C + 2) * 8;
};

// One Stockham stage of radix R over C columns of length L in shared memory (pitch C), or from
// global memory for the first stage.  Each thread owns 8 values (8 / R work items).  The stage
// reads everything it needs into registers, the CTA synchronises, then it writes: the buffer is
// updated in place.  Work item w -> column c = w % C, j = w / C; Stockham DIT: inputs at
// j + r L/R, twiddle w_L^(r (j mod Ns) L/(Ns R)), outputs at (j/Ns) Ns R + j mod Ns + r Ns.
template <int LOGL, int R>
__device__ __forceinline__ void col_stage(u64* s, const u64* twL, unsigned Ns, u64 (&v)[8],
                                          bool from_global, const u64* __restrict__ gsrc,
                                          size_t ld_in, size_t n_valid, unsigned c0,
                                          bool last_padded) {
  constexpr int L = ColCfg<LOGL>::L, C = ColCfg<LOGL>::C, T = ColCfg<LOGL>::T;
  constexpr int ITEMS = 8 / R;
  constexpr int NW = C * L / R;
#pragma unroll
  for (int it = 0; it < ITEMS; ++it) {
    const unsigned w = threadIdx.x + it * T;
    if (w < NW) {
      const unsigned c = w % C, j = w / C;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const unsigned row = j + r * (L / R);
        u64 x;
        if (from_global) {
          size_t e = (size_t)row * ld_in + c0 + c;
          x = e < n_valid ? gl_canon(__ldg(gsrc + e)) : 0;
        } else {
          x = s[row * C + c];
        }
        v[it * R + r] = x;
      }
      if (Ns > 1) {
        const unsigned k = j % Ns, step = k * (L / (Ns * R));
#pragma unroll
        for (int r = 1; r < R; ++r) v[it * R + r] = gl_mul(v[it * R + r], twL[r * step]);
      }
      dft_small<R>(&v[it * R]);
    }
  }
  __syncthreads();
  const unsigned pitch = last_padded ? C + 1 : C;
#pragma unroll
  for (int it = 0; it < ITEMS; ++it) {
    const unsigned w = threadIdx.x + it * T;
    if (w < NW) {
      const unsigned c = w % C, j = w / C;
      const unsigned k = j % Ns, idxD = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[(idxD + r * Ns) * pitch + c] = v[it * R + r];
    }
  }
  __syncthreads();
}

// Transform C consecutive columns (c0 ..) of a row-major matrix (row stride ld_in, L rows,
// entries at or beyond n_valid read as zero) of vector blockIdx.y.
// TRANSPOSED: out[b*obs + (c0+c)*L + j] = X_c[j] * w_N^(j (c0+c))   (four-step pass A)
// otherwise:  out[b*obs + j*ld_out + c0 + c] = X_c[j]                (four-step pass B)
template <int LOGL, bool TRANSPOSED>
__global__ void __launch_bounds__(ColCfg<LOGL>::T)
    ntt_col_kernel(const u64* __restrict__ in, size_t ibs, size_t ld_in, size_t n_valid,
                   u64* __restrict__ out, size_t obs, size_t ld_out, unsigned logN,
                   const u64* __restrict__ tw) {
  constexpr int L = ColCfg<LOGL>::L, C = ColCfg<LOGL>::C, T = ColCfg<LOGL>::T;
  extern __shared__ u64 sm[];
  u64* twL = sm;
  u64* s = sm + L;
  const size_t b = blockIdx.y;
  const unsigned c0 = blockIdx.x * C;
  for (unsigned e = threadIdx.x; e < (unsigned)L; e += T) twL[e] = __ldg(tw + ((size_t)e << (TW_LOG - LOGL)));
  __syncthreads();
  const u64* src = in + b * ibs;
  u64 v[8];
  constexpr int S8 = LOGL / 3, REM = LOGL % 3;
  constexpr int NST = S8 + (REM ? 1 : 0);
  unsigned Ns = 1;
  int st = 0;
#pragma unroll
  for (int q = 0; q < S8; ++q, ++st) {
    col_stage<LOGL, 8>(s, twL, Ns, v, st == 0, src, ld_in, n_valid, c0, TRANSPOSED && st == NST - 1);
    Ns *= 8;
  }
  if (REM == 2) col_stage<LOGL, 4>(s, twL, Ns, v, st == 0, src, ld_in, n_valid, c0, TRANSPOSED);
  if (REM == 1) col_stage<LOGL, 2>(s, twL, Ns, v, st == 0, src, ld_in, n_valid, c0, TRANSPOSED);
  u64* dst = out + b * obs;
  if (TRANSPOSED) {
    const unsigned shift = TW_LOG - logN;
    const size_t mask = ((size_t)1 << logN) - 1;
    for (unsigned idx = threadIdx.x; idx < (unsigned)(C * L); idx += T) {
      const unsigned j = idx % L, c = idx / L;
      u64 x = s[j * (C + 1) + c];
      const size_t e = ((size_t)j * (c0 + c)) & mask;
      if (e) x = gl_mul(x, __ldg(tw + (e << shift)));
      dst[(size_t)(c0 + c) * L + j] = x;
    }
  } else {
    for (unsigned idx = threadIdx.x; idx < (unsigned)(C * L); idx += T) {
      const unsigned c = idx % C, j = idx / C;
      dst[(size_t)j * ld_out + c0 + c] = s[j * C + c];
    }
  }
}

template <int LOGL, bool TR>
void launch_col(const u64* in, size_t ibs, size_t ld_in, size_t n_valid, u64* out, size_t obs,
                size_t ld_out, unsigned logN, size_t ncols, size_t batch, const u64* tw,
                cudaStream_t st) {
  using Cfg = ColCfg<LOGL>;
  if (ncols % Cfg::C) throw ShapeError("ntt: column count not a multiple of the tile");
  auto k = ntt_col_kernel<LOGL, TR>;
  LGS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM));
  dim3 grid((unsigned)(ncols / Cfg::C), (unsigned)batch);
  k<<<grid, Cfg::T, Cfg::SMEM, st>>>(in, ibs, ld_in, n_valid, out, obs, ld_out, logN, tw);
  LGS_LAUNCH_CHECK();
}

template <bool TR>
void launch_col_dispatch(unsigned logL, const u64* in, size_t ibs, size_t ld_in, size_t n_valid,
                         u64* out, size_t obs, size_t ld_out, unsigned logN, size_t ncols,
                         size_t batch, const u64* tw, cudaStream_t st) {
  switch (logL) {
#define LGS_COL_CASE(K) \
  case K: launch_col<K, TR>(in, ibs, ld_in, n_valid, out, obs, ld_out, logN, ncols, batch, tw, st); break;
    LGS_COL_CASE(3) LGS_COL_CASE(4) LGS_COL_CASE(5) LGS_COL_CASE(6) LGS_COL_CASE(7)
    LGS_COL_CASE(8) LGS_COL_CASE(9) LGS_COL_CASE(10) LGS_COL_CASE(11)
#undef LGS_COL_CASE
    default: throw ShapeError("ntt: unsupported sub-transform size");
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
  if (logN > 22) throw ShapeError("ntt: transforms above 2^22 are not supported");
  // four-step: x[k1 N2 + k2]; pass A transforms columns k2 (length N1) into Z[k2][j1] with the
  // twiddle w_N^(j1 k2); pass B transforms columns j1 of Z (length N2) into X[j1 + N1 j2].
  const unsigned logN1 = (logN + 1) / 2, logN2 = logN - logN1;
  const size_t N1 = (size_t)1 << logN1, N2 = (size_t)1 << logN2;
  launch_col_dispatch<true>(logN1, in, in_stride, N2, n_in, scratch, N, N1, logN, N2, batch, tw, st);
  launch_col_dispatch<false>(logN2, scratch, N, N1, N, out, out_stride, N1, logN, N1, batch, tw, st);
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
