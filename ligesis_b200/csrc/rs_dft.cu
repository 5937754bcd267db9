// Batched Reed-Solomon encoding of the commitment rows: out[j] = sum_k in[k] g_N^(jk) for every
// row (p3-dft's `Radix2Dit::dft` in natural order, pcs/src/ligesis.rs:222-235), for
// N = 2^14 .. 2^18 with the row either zero-padded from N/2 values (rate 1/2) or full.
//
// Four-step split N = 4096 * N2, k = k1 N2 + k2, j = j1 + 4096 j2:
//   X[j1 + 4096 j2] = sum_k2 w_N2^(j2 k2) w_N^(j1 k2) sum_k1 x[k1 N2 + k2] w_4096^(j1 k1)
// pass A  one CTA per (row, 4 consecutive columns k2): the 4096-point column DFTs over k1 as
//         64 x 64, each 64-point DFT as radix-8 x radix-8 shared by 8 warps (one radix-8 per
//         thread, a shared-memory exchange between the two), written as Z[k2][j1] (contiguous
//         in j1).  Global reads are 32-byte runs; the zero half of a rate-1/2 row is never read.
// pass B  the four-step twiddle w_N^(j1 k2) from a table laid out [k2][j1], then the N2-point
//         DFT over k2 (N2 = 64: 8 warps on 32 columns the same way; smaller N2: one thread per
//         column, in registers); reads Z and writes X in 256-byte runs per warp.
// Inside a radix-8 the twiddles are 8th roots of unity, powers of two (2^120 is the order-8 root
// of the reference's generator), so they are shifts; the twiddles between the radix-8 digits
// are per-warp constants or table entries and use the carry-chain multiplication.
#include "kernels.cuh"

namespace lgs {

namespace {

// (lo + hi 2^64) mod p for hi < 2^32: 2^64 = 2^32 - 1, so this is lo + (hi << 32) - hi, which
// overflows at most once.
__device__ __forceinline__ u64 reduce_hi32(u64 lo, u64 hi) {
  const u64 t = (hi << 32) - hi;
  u64 s = lo + t;
  if (s < t) s += GL_EPS;
  return s >= GL_P ? s - GL_P : s;
}

// x * 2^S mod p for a compile-time S; x canonical, result canonical.  2^96 = -1 mod p.
template <unsigned S>
__device__ __forceinline__ u64 rot(u64 x) {
  constexpr unsigned s = S % 192;
  if constexpr (s == 0) {
    return x;
  } else if constexpr (s >= 96) {
    return gl_neg(rot<s - 96>(x));
  } else if constexpr (s < 32) {
    return reduce_hi32(x << s, x >> (64 - s));
  } else if constexpr (s < 64) {
    return gl_reduce(x << s, x >> (64 - s));
  } else {
    // x = xl + 2^32 xh; 2^64 = 2^32 - 1 and 2^96 = -1 give
    // x 2^s = xl 2^(s-32) - (xl + xh) 2^(s-64): one 96-bit reduction and a subtraction.
    const u64 xl = x & GL_EPS, xh = x >> 32;
    const u64 a = reduce_hi32(xl << (s - 32), xl >> (96 - s));
    u64 b = (xl + xh) << (s - 64);  // < 2^64
    if (b >= GL_P) b -= GL_P;
    return gl_sub(a, b);
  }
}

// (a, b) <- (a + 2^S b, a - 2^S b); a negative power (S mod 192 >= 96) swaps the add and sub.
template <unsigned S>
__device__ __forceinline__ void bfly(u64& a, u64& b) {
  constexpr unsigned s = S % 192;
  if constexpr (s >= 96) {
    const u64 t = rot<s - 96>(b);
    b = gl_add(a, t);
    a = gl_sub(a, t);
  } else {
    const u64 t = rot<s>(b);
    b = gl_sub(a, t);
    a = gl_add(a, t);
  }
}

// log2 of g_t (the reference generator's order-2^t root) as a power of two: g_t = 2^E mod p.
template <int T>
struct RootLog;
template <> struct RootLog<2> { static constexpr unsigned E = 48; };
template <> struct RootLog<3> { static constexpr unsigned E = 120; };
template <> struct RootLog<4> { static constexpr unsigned E = 156; };
template <> struct RootLog<5> { static constexpr unsigned E = 78; };

// Natural-order R-point DFTs (R = 2, 4, 8) on registers v[0], v[ST], ..., v[(R-1) ST];
// radix-2 DIT on the bit-reversed inputs.  ZH: the upper half of the inputs is zero.
template <int ST, bool ZH>
__device__ __forceinline__ void dft_r2(u64* v) {
  if constexpr (ZH) {
    v[ST] = v[0];
  } else {
    bfly<0>(v[0], v[ST]);
  }
}
template <int ST, bool ZH>
__device__ __forceinline__ void dft_r4(u64* v) {
  u64 a0 = v[0], a1 = v[2 * ST], a2 = v[ST], a3 = v[3 * ST];
  if constexpr (ZH) {
    a1 = a0;
    a3 = a2;
  } else {
    bfly<0>(a0, a1);
    bfly<0>(a2, a3);
  }
  bfly<0>(a0, a2);
  bfly<RootLog<2>::E>(a1, a3);
  v[0] = a0, v[ST] = a1, v[2 * ST] = a2, v[3 * ST] = a3;
}

template <int ST, bool ZH>
__device__ __forceinline__ void dft_r8(u64* v) {
  // bit-reversed pairs (0,4) (2,6) (1,5) (3,7)
  u64 a0 = v[0], a1 = v[4 * ST], a2 = v[2 * ST], a3 = v[6 * ST];
  u64 a4 = v[ST], a5 = v[5 * ST], a6 = v[3 * ST], a7 = v[7 * ST];
  if constexpr (ZH) {
    a1 = a0, a3 = a2, a5 = a4, a7 = a6;
  } else {
    bfly<0>(a0, a1);
    bfly<0>(a2, a3);
    bfly<0>(a4, a5);
    bfly<0>(a6, a7);
  }
  constexpr unsigned W8 = RootLog<3>::E, W4 = RootLog<2>::E;
  bfly<0>(a0, a2);
  bfly<W4>(a1, a3);
  bfly<0>(a4, a6);
  bfly<W4>(a5, a7);
  bfly<0>(a0, a4);
  bfly<W8>(a1, a5);
  bfly<2 * W8>(a2, a6);
  bfly<3 * W8>(a3, a7);
  v[0] = a0, v[ST] = a1, v[2 * ST] = a2, v[3 * ST] = a3;
  v[4 * ST] = a4, v[5 * ST] = a5, v[6 * ST] = a6, v[7 * ST] = a7;
}

// In-register DFT of L = 2^LOGL <= 64 natural-order values; ZH: v[L/2 ..] are zero.  The result
// Y[j] is left in v[Pos<LOGL>::at(j)].
template <int LOGL>
struct Pos {
  static constexpr int A = LOGL <= 3 ? (1 << LOGL) : (LOGL == 4 ? 4 : 8);
  static constexpr int B = (1 << LOGL) / A;
  static __host__ __device__ constexpr int at(int j) {
    return LOGL <= 3 ? j : A * (j % B) + j / B;
  }
};

template <int R, bool ZH, int ST>
__device__ __forceinline__ void dft_any(u64* v) {
  if constexpr (R == 8) dft_r8<ST, ZH>(v);
  else if constexpr (R == 4) dft_r4<ST, ZH>(v);
  else dft_r2<ST, ZH>(v);
}

// L = A * B, k = ka + A kb, j = jb + B ja:
//   Y[jb + B ja] = sum_ka w_A^(ja ka) w_L^(jb ka) sum_kb v[ka + A kb] w_B^(jb kb)
// step 1: the B-point DFTs over kb; step 2: the twiddles w_L^(jb ka) (powers of two);
// step 3: the A-point DFTs over ka.
template <int A, int B, bool ZH, unsigned EL, int KA>
__device__ __forceinline__ void step1(u64* v) {
  if constexpr (KA < A) {
    dft_any<B, ZH, A>(v + KA);
    step1<A, B, ZH, EL, KA + 1>(v);
  }
}
template <int A, int B, unsigned EL, int KA, int JB>
__device__ __forceinline__ void step2(u64* v) {
  if constexpr (KA < A) {
    if constexpr (JB < B) {
      v[KA + A * JB] = rot<(EL * KA * JB) % 192>(v[KA + A * JB]);
      step2<A, B, EL, KA, JB + 1>(v);
    } else {
      step2<A, B, EL, KA + 1, 0>(v);
    }
  }
}
template <int A, int B, int JB>
__device__ __forceinline__ void step3(u64* v) {
  if constexpr (JB < B) {
    dft_any<A, false, 1>(v + A * JB);
    step3<A, B, JB + 1>(v);
  }
}

template <int LOGL, bool ZH>
__device__ __forceinline__ void dft64(u64* v) {
  if constexpr (LOGL <= 3) {
    dft_any<(1 << LOGL), ZH, 1>(v);
  } else {
    constexpr int A = Pos<LOGL>::A, B = Pos<LOGL>::B;
    step1<A, B, ZH, RootLog<LOGL>::E, 0>(v);
    step2<A, B, RootLog<LOGL>::E, 1, 1>(v);
    step3<A, B, 0>(v);
  }
}

// ---- pass A: the 4096-point column DFTs of 4 columns, 16 warps in two groups of 8 ------------
// k1 = a + 64 b, a = a0 + 8 a1, b = b0 + 8 b1 (all digits < 8).  Phase 1, per group round:
// 32 lane-columns (c, a) with lane = c + 4 (a mod 8); warp w holds b0 = w and does the radix-8
// over b1, multiplies by w_64^(jb1 b0), and exchanges through shared memory so that warp w then
// holds jb1 = w and does the radix-8 over b0: j' = jb1 + 8 jb0 is the 64-point output over b.
// After the w_4096^(j' a) twiddle the values go to the column tile big[c][j'][a].  Phase 2 does
// the same over a for lane-columns (c, j') and writes Z[k2][j1], j1 = j' + 64 (ja1 + 8 ja0).
constexpr int PA_THREADS = 512;
constexpr int PA_COLS = 4;
constexpr int PA_JS = 65;    // big[] stride of j' (odd: conflict-free phase-2 reads)
constexpr int PA_CS = 4164;  // big[] stride of a column (= 4 mod 16: conflict-free phase-1 stores)
constexpr size_t PA_SMEM = ((size_t)PA_COLS * PA_CS + 2 * 2048) * 8;

__device__ __forceinline__ void group_sync(unsigned grp) {
  asm volatile("bar.sync %0, 256;" ::"r"(1 + grp) : "memory");
}

template <bool HALF>
__global__ void __launch_bounds__(PA_THREADS, 1)
    rs_pass_a_kernel(const u64* __restrict__ in, size_t ld_in, u64* __restrict__ z, unsigned N2,
                     const u64* __restrict__ tw4096) {
  extern __shared__ u64 sm[];
  u64* big = sm;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned grp = warp >> 3, w = warp & 7;
  u64* ex = sm + PA_COLS * PA_CS + grp * 2048;  // [jb][w][lane]
  const size_t row = blockIdx.y;
  const unsigned k2_0 = blockIdx.x * PA_COLS;
  u64 t64[8];  // w_64^(j w) = w_4096^(64 j w), the same for the whole warp
#pragma unroll
  for (int j = 1; j < 8; ++j) t64[j] = __ldg(tw4096 + 64 * j * w);

  // phase 1 inputs of this thread's four rounds, loaded up front
  constexpr int NB1 = HALF ? 4 : 8;
  const unsigned c = lane & 3;
  u64 pre[4][NB1];
  {
    const u64* src = in + row * ld_in + k2_0 + c;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const unsigned a = 8 * (grp + 2 * i) + (lane >> 2);
      const u64* s = src + (size_t)(a + 64 * w) * N2;
#pragma unroll
      for (int b1 = 0; b1 < NB1; ++b1) pre[i][b1] = gl_canon(__ldg(s + (size_t)b1 * 512 * N2));
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const unsigned a = 8 * (grp + 2 * i) + (lane >> 2);
    u64 v[8];
#pragma unroll
    for (int b1 = 0; b1 < 8; ++b1) v[b1] = b1 < NB1 ? pre[i][b1 < NB1 ? b1 : 0] : 0;
    dft_r8<1, HALF>(v);
#pragma unroll
    for (int j = 1; j < 8; ++j) v[j] = gl_mul(v[j], t64[j]);
#pragma unroll
    for (int j = 0; j < 8; ++j) ex[(j * 8 + w) * 32 + lane] = v[j];
    group_sync(grp);
#pragma unroll
    for (int b0 = 0; b0 < 8; ++b0) v[b0] = ex[(w * 8 + b0) * 32 + lane];
    dft_r8<1, false>(v);
#pragma unroll
    for (int j0 = 0; j0 < 8; ++j0) {
      const unsigned jp = w + 8 * j0;
      v[j0] = gl_mul(v[j0], __ldg(tw4096 + jp * a));
      big[c * PA_CS + jp * PA_JS + a] = v[j0];
    }
    group_sync(grp);
  }
  __syncthreads();
#pragma unroll 1
  for (unsigned r = grp; r < 8; r += 2) {
    const unsigned cc = r >> 1, jp = 32 * (r & 1) + lane;
    u64 v[8];
    const u64* s = big + cc * PA_CS + jp * PA_JS + w;
#pragma unroll
    for (int a1 = 0; a1 < 8; ++a1) v[a1] = s[8 * a1];
    dft_r8<1, false>(v);
#pragma unroll
    for (int j = 1; j < 8; ++j) v[j] = gl_mul(v[j], t64[j]);
#pragma unroll
    for (int j = 0; j < 8; ++j) ex[(j * 8 + w) * 32 + lane] = v[j];
    group_sync(grp);
#pragma unroll
    for (int a0 = 0; a0 < 8; ++a0) v[a0] = ex[(w * 8 + a0) * 32 + lane];
    dft_r8<1, false>(v);
    u64* dst = z + (row * N2 + k2_0 + cc) * 4096 + jp;
#pragma unroll
    for (int j0 = 0; j0 < 8; ++j0) dst[64 * (w + 8 * j0)] = v[j0];
    group_sync(grp);
  }
}

// ---- pass B for N2 = 64: 8 warps on 32 consecutive j1 of one row ------------------------------
// k2 = ka + 8 kb: warp w = ka loads Z[k2][j1] (256-byte rows), applies w_N^(j1 k2), does the
// radix-8 over kb, multiplies by w_64^(jb ka), exchanges, and as jb = w does the radix-8 over ka.
__global__ void __launch_bounds__(256)
    rs_pass_b64_kernel(const u64* __restrict__ z, u64* __restrict__ out, size_t ld_out,
                       const u64* __restrict__ t4, const u64* __restrict__ tw4096) {
  __shared__ u64 ex[8 * 8 * 32];
  const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned j1 = blockIdx.x * 32 + lane;
  const size_t row = blockIdx.y;
  const u64* src = z + row * ((size_t)64 * 4096) + j1;
  u64 v[8];
#pragma unroll
  for (int kb = 0; kb < 8; ++kb) v[kb] = src[(size_t)(w + 8 * kb) * 4096];
#pragma unroll
  for (int kb = 0; kb < 8; ++kb) v[kb] = gl_mul(v[kb], __ldg(t4 + (w + 8 * kb) * 4096 + j1));
  dft_r8<1, false>(v);
#pragma unroll
  for (int j = 1; j < 8; ++j) v[j] = gl_mul(v[j], __ldg(tw4096 + 64 * j * w));
#pragma unroll
  for (int j = 0; j < 8; ++j) ex[(j * 8 + w) * 32 + lane] = v[j];
  __syncthreads();
#pragma unroll
  for (int ka = 0; ka < 8; ++ka) v[ka] = ex[(w * 8 + ka) * 32 + lane];
  dft_r8<1, false>(v);
  u64* dst = out + row * ld_out + j1;
#pragma unroll
  for (int j0 = 0; j0 < 8; ++j0) dst[(size_t)(w + 8 * j0) * 4096] = v[j0];
}

constexpr int PB_THREADS = 128;

template <int LOGL>
__global__ void __launch_bounds__(PB_THREADS)
    rs_pass_b_kernel(const u64* __restrict__ z, u64* __restrict__ out, size_t ld_out,
                     const u64* __restrict__ t4) {
  constexpr int L = 1 << LOGL;
  const unsigned j1 = blockIdx.x * PB_THREADS + threadIdx.x;
  const size_t row = blockIdx.y;
  const u64* src = z + row * ((size_t)L * 4096) + j1;
  u64 r[L];
#pragma unroll
  for (int k2 = 0; k2 < L; ++k2) r[k2] = src[(size_t)k2 * 4096];
#pragma unroll
  for (int k2 = 1; k2 < L; ++k2) r[k2] = gl_mul(r[k2], __ldg(t4 + k2 * 4096 + j1));
  dft64<LOGL, false>(r);
  u64* dst = out + row * ld_out + j1;
#pragma unroll
  for (int j2 = 0; j2 < L; ++j2) dst[(size_t)j2 * 4096] = r[Pos<LOGL>::at(j2)];
}

// tables[0 .. 4096) = w_4096^e; the four-step table of each logN at rs_table_offset(logN):
// T[k2 * 4096 + j1] = w_N^(j1 k2) for k2 < N / 4096.
__global__ void rs_tables_kernel(u64* tables, const u64* __restrict__ tw, size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  if (i < 4096) {
    tables[i] = tw[i << (TW_LOG - 12)];
    return;
  }
  unsigned logN = RS_LOGN_MIN;
  size_t off = 4096;
  while (off + ((size_t)1 << logN) <= i) off += (size_t)1 << logN++;
  const size_t e = i - off, k2 = e >> 12, j1 = e & 4095;
  tables[i] = tw[(j1 * k2) << (TW_LOG - logN)];
}

template <bool HALF>
void launch_a(const u64* in, size_t ld_in, u64* z, unsigned N2, size_t rows, const u64* tw4096,
              cudaStream_t st) {
  auto k = rs_pass_a_kernel<HALF>;
  LGS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PA_SMEM));
  dim3 grid(N2 / PA_COLS, (unsigned)rows);
  k<<<grid, PA_THREADS, PA_SMEM, st>>>(in, ld_in, z, N2, tw4096);
  LGS_LAUNCH_CHECK();
}

template <int LOGL>
void launch_b(const u64* z, u64* out, size_t ld_out, size_t rows, const u64* t4, cudaStream_t st) {
  dim3 grid(4096 / PB_THREADS, (unsigned)rows);
  rs_pass_b_kernel<LOGL><<<grid, PB_THREADS, 0, st>>>(z, out, ld_out, t4);
  LGS_LAUNCH_CHECK();
}

// ---- the arithmetic floor of the encoding: its operations with no memory traffic -------------
// op 0: one radix-8 DFT (dft_r8, as every stage of both passes) per iteration; op 1: eight
// independent twiddle multiplications (gl_mul) per iteration.  Eight values per thread, a
// checksum to `sink` so nothing is optimised away.
__global__ void __launch_bounds__(256) rs_alu_floor_kernel(unsigned iters, int op, u64* sink) {
  const u64 seed = 0x9E3779B97F4A7C15ull * (blockIdx.x * blockDim.x + threadIdx.x + 1);
  u64 v[8], t[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    v[j] = gl_canon(seed + 0x632BE59BD9B4E019ull * j);
    t[j] = gl_canon(seed ^ (0xD1B54A32D192ED03ull * (j + 3)));
  }
  if (op == 0) {
#pragma unroll 1
    for (unsigned i = 0; i < iters; ++i) dft_r8<1, false>(v);
  } else {
#pragma unroll 1
    for (unsigned i = 0; i < iters; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = gl_mul(v[j], t[j]);
  }
  u64 acc = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) acc ^= v[j];
  if (acc == 0x0123456789ABCDEFull) *sink = acc;  // practically never: keeps v live
}

}  // namespace

double rs_alu_rate(int op, unsigned iters, u64* sink, cudaStream_t st) {
  int dev = 0, sms = 0;
  LGS_CUDA(cudaGetDevice(&dev));
  LGS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int per_sm = 1;
  LGS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rs_alu_floor_kernel, 256, 0));
  const unsigned blocks = (unsigned)(sms * std::max(1, per_sm));
  cudaEvent_t e0, e1;
  LGS_CUDA(cudaEventCreate(&e0));
  LGS_CUDA(cudaEventCreate(&e1));
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {  // the first launch warms up; keep the best
    LGS_CUDA(cudaEventRecord(e0, st));
    rs_alu_floor_kernel<<<blocks, 256, 0, st>>>(iters, op, sink);
    LGS_LAUNCH_CHECK();
    LGS_CUDA(cudaEventRecord(e1, st));
    LGS_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    LGS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double ops = (double)blocks * 256 * iters * (op == 0 ? 1.0 : 8.0);
    if (rep > 0 && ms > 0) best = std::max(best, ops / (ms * 1e-3));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

size_t rs_table_offset(unsigned logN) {
  size_t off = 4096;
  for (unsigned l = RS_LOGN_MIN; l < logN; ++l) off += (size_t)1 << l;
  return off;
}
size_t rs_tables_elems() { return rs_table_offset(RS_LOGN_MAX + 1); }

void build_rs_tables(u64* tables, const u64* tw, cudaStream_t st) {
  const size_t total = rs_tables_elems();
  rs_tables_kernel<<<cdiv(total, 256), 256, 0, st>>>(tables, tw, total);
  LGS_LAUNCH_CHECK();
}

bool rs_dft_supported(unsigned logN, size_t n_in) {
  const size_t N = (size_t)1 << logN;
  return logN >= RS_LOGN_MIN && logN <= RS_LOGN_MAX && (2 * n_in == N || n_in == N);
}

void rs_dft_rows(const u64* in, size_t ld_in, size_t n_in, u64* out, size_t ld_out,
                 unsigned logN, size_t rows, u64* z, const u64* tables, cudaStream_t st) {
  if (!rs_dft_supported(logN, n_in)) throw ShapeError("rs_dft_rows: unsupported size");
  if (rows == 0) return;
  if (rows > 65535) throw ShapeError("rs_dft_rows: too many rows");
  const size_t N = (size_t)1 << logN;
  const unsigned N2 = (unsigned)(N >> 12);
  if (2 * n_in == N)
    launch_a<true>(in, ld_in, z, N2, rows, tables, st);
  else
    launch_a<false>(in, ld_in, z, N2, rows, tables, st);
  const u64* t4 = tables + rs_table_offset(logN);
  switch (logN - 12) {
    case 2: launch_b<2>(z, out, ld_out, rows, t4, st); break;
    case 3: launch_b<3>(z, out, ld_out, rows, t4, st); break;
    case 4: launch_b<4>(z, out, ld_out, rows, t4, st); break;
    case 5: launch_b<5>(z, out, ld_out, rows, t4, st); break;
    case 6: {
      dim3 grid(4096 / 32, (unsigned)rows);
      rs_pass_b64_kernel<<<grid, 256, 0, st>>>(z, out, ld_out, t4, tables);
      LGS_LAUNCH_CHECK();
      break;
    }
    default: throw ShapeError("rs_dft_rows: unsupported size");
  }
}

}  // namespace lgs
