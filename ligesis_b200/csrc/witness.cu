// proofsys' rescaled linear-layer witness on the device (proofsys/src/model.rs:360-361 and the
// integer kernels of proofsys/src/tensor.rs): Q, REM = floor_div(X W, divisor) with REM in
// [0, divisor), Y = Q + bias, and Y lifted to Goldilocks like encode_i64
// (proofsys/src/witness.rs:102-108).  The reference multiplies i64 matrices with i128
// accumulators and panics when a result leaves the i64 range; this kernel does the same products
// exactly (128-bit accumulators) and reports such a result as an error instead.
//
// The values are fixed-point integers (scale 2^12, activations up to about 2^20), not int8: a
// 32 x 64 output tile per CTA, 16 x 16 threads with a 2 x 4 block each, the K dimension staged
// through shared memory 32 at a time.  Each stage sums in the cheapest exact arithmetic its
// operands allow (fused multiply-adds of doubles while every partial sum stays below 2^53, else
// 64-bit or 128-bit integer sums) and adds the stage sum to exact 128-bit (hi, lo) accumulators.
// GPT-2's layers have 31 rows, so K is split over CTAs to fill the GPU and the exact partial sums
// are added by a second kernel.  The largest layer, the vocabulary head (31 x 768 x 50257), is
// 1.2 G products.
#include <algorithm>
#include <cstring>

#include "prover.cuh"
#include "witness.cuh"

namespace lgs {

namespace {

constexpr int LW_TM = 32, LW_TN = 64, LW_K = 32;  // output tile rows x cols, K per stage
constexpr size_t LW_XS_BYTES = (size_t)LW_K * (LW_TM + 1) * 8;
constexpr size_t LW_WS_BYTES = (size_t)LW_K * (LW_TN + 1) * 8;
constexpr size_t LW_SMEM = 2 * (LW_XS_BYTES + LW_WS_BYTES) + 4 * 8;

struct LwArgs {
  const int64_t* x;
  const int64_t* w;
  const int64_t* bias;
  size_t rows, inner, cols, kchunk;
  int64_t d;
  int wt;
  Acc128* part;  // [split][rows][cols] when split over K
  int64_t *q, *rem, *y;
  uint64_t* yf;
  int* err;
};

__device__ __forceinline__ uint64_t mag64(int64_t v) {
  return v < 0 ? ~(uint64_t)v + 1 : (uint64_t)v;  // |v| (2^63 at INT64_MIN)
}
__device__ __forceinline__ int bitlen64(uint64_t v) { return 64 - __clzll((long long)v); }
// s += x * y for 32-bit signed x, y: one wide multiply-add into the 64-bit sum.
__device__ __forceinline__ void mad_wide(int64_t& s, int32_t x, int32_t y) {
  asm("mad.wide.s32 %0, %1, %2, %0;" : "+l"(s) : "r"(x), "r"(y));
}

// The K loop of a tile.  Each stage of LW_K values picks its own exact arithmetic from the
// largest |x| and |w| it has just staged (an OR of their magnitudes, gathered in shared memory),
// so no separate pass over the operands is needed:
//   bx + bw + log2 LW_K <= 53: fused multiply-adds of doubles (exact: every intermediate is an
//     integer below 2^53), one instruction per product;
//   bx + bw + log2 LW_K <= 62 and both <= 31 bits: 32-bit products summed in 64 bits;
//   bx + bw + log2 LW_K <= 62: 64-bit products summed in 64 bits;
//   otherwise: 128-bit sums of the 64-bit products.
// A stage's sum is exact and is added to the 128-bit accumulator.
__device__ __forceinline__ void lw_tile_loop(const LwArgs& a, int64_t (*xs)[LW_TM + 1],
                                             int64_t (*ws)[LW_TN + 1], double (*xd)[LW_TM + 1],
                                             double (*wd)[LW_TN + 1],
                                             unsigned long long (*mags)[2], size_t r0, size_t c0,
                                             size_t kb, size_t ke, Acc128 (&acc)[2][4]) {
  const unsigned tx = threadIdx.x & 15, ty = threadIdx.x >> 4, lane = threadIdx.x & 31;
  // Each of the 256 threads stages 4 values of x and 8 of w per stage (LW_TM x LW_K and
  // LW_TN x LW_K).  The next stage's values are loaded into registers before this stage's
  // arithmetic, so their global-memory latency is hidden behind it.
  constexpr int NX = LW_TM * LW_K / 256, NW = LW_TN * LW_K / 256;
  int64_t vx[NX], vw[NW];
  auto x_slot = [&](int i, unsigned& rr, unsigned& kk) {
    const unsigned e = threadIdx.x + 256 * i;
    rr = e / LW_K;
    kk = e % LW_K;
  };
  auto w_slot = [&](int i, unsigned& cc, unsigned& kk) {
    const unsigned e = threadIdx.x + 256 * i;
    if (a.wt) {  // w is cols x inner: consecutive threads read consecutive k
      cc = e / LW_K;
      kk = e % LW_K;
    } else {  // w is inner x cols: consecutive threads read consecutive columns
      kk = e / LW_TN;
      cc = e % LW_TN;
    }
  };
  auto fetch = [&](size_t k0) {
#pragma unroll
    for (int i = 0; i < NX; ++i) {
      unsigned rr, kk;
      x_slot(i, rr, kk);
      const size_t gr = r0 + rr, gk = k0 + kk;
      vx[i] = (gr < a.rows && gk < ke) ? a.x[gr * a.inner + gk] : 0;
    }
#pragma unroll
    for (int i = 0; i < NW; ++i) {
      unsigned cc, kk;
      w_slot(i, cc, kk);
      const size_t gc = c0 + cc, gk = k0 + kk;
      int64_t v = 0;
      if (gc < a.cols && gk < ke) v = a.wt ? a.w[gc * a.inner + gk] : a.w[gk * a.cols + gc];
      vw[i] = v;
    }
  };
  fetch(kb);
  unsigned par = 0;
  for (size_t k0 = kb; k0 < ke; k0 += LW_K, par ^= 1) {
    uint64_t ox = 0, ow = 0;
#pragma unroll
    for (int i = 0; i < NX; ++i) {
      unsigned rr, kk;
      x_slot(i, rr, kk);
      xs[kk][rr] = vx[i];
      xd[kk][rr] = (double)vx[i];
      ox |= mag64(vx[i]);
    }
#pragma unroll
    for (int i = 0; i < NW; ++i) {
      unsigned cc, kk;
      w_slot(i, cc, kk);
      ws[kk][cc] = vw[i];
      wd[kk][cc] = (double)vw[i];
      ow |= mag64(vw[i]);
    }
    if (k0 + LW_K < ke) fetch(k0 + LW_K);
    // OR over the warp (two 32-bit halves), then over the CTA into this stage's slot
    const unsigned xl = __reduce_or_sync(0xffffffffu, (unsigned)ox);
    const unsigned xh = __reduce_or_sync(0xffffffffu, (unsigned)(ox >> 32));
    const unsigned wl = __reduce_or_sync(0xffffffffu, (unsigned)ow);
    const unsigned wh = __reduce_or_sync(0xffffffffu, (unsigned)(ow >> 32));
    if (lane == 0) {
      atomicOr(&mags[par][0], ((unsigned long long)xh << 32) | xl);
      atomicOr(&mags[par][1], ((unsigned long long)wh << 32) | wl);
    }
    __syncthreads();
    const int bx = bitlen64(mags[par][0]), bw = bitlen64(mags[par][1]);
    // the other slot was last read before this barrier and is next written after the next one
    if (threadIdx.x == 0) mags[par ^ 1][0] = mags[par ^ 1][1] = 0;
    if (bx + bw + 5 <= 53) {  // 2^5 = LW_K products per sum
      // every product and partial sum is an integer below 2^53 in magnitude, so each fused
      // multiply-add of doubles is exact (no rounding ever happens)
      double d[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll 8
      for (int kk = 0; kk < LW_K; ++kk) {
        const double x0 = xd[kk][2 * ty], x1 = xd[kk][2 * ty + 1];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const double b = wd[kk][tx + 16 * j];
          d[0][j] = __fma_rn(x0, b, d[0][j]);
          d[1][j] = __fma_rn(x1, b, d[1][j]);
        }
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int64_t v = __double2ll_rn(d[i][j]);
          add128(acc[i][j], Acc128{(uint64_t)v, (uint64_t)(v >> 63)});
        }
    } else if (bx + bw + 5 <= 62) {
      int64_t s64[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
      if (bx <= 31 && bw <= 31) {
#pragma unroll 8
        for (int kk = 0; kk < LW_K; ++kk) {
          const int32_t x0 = (int32_t)xs[kk][2 * ty], x1 = (int32_t)xs[kk][2 * ty + 1];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int32_t b = (int32_t)ws[kk][tx + 16 * j];
            mad_wide(s64[0][j], x0, b);
            mad_wide(s64[1][j], x1, b);
          }
        }
      } else {
#pragma unroll 8
        for (int kk = 0; kk < LW_K; ++kk) {
          const int64_t x0 = xs[kk][2 * ty], x1 = xs[kk][2 * ty + 1];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int64_t b = ws[kk][tx + 16 * j];
            s64[0][j] += x0 * b;
            s64[1][j] += x1 * b;
          }
        }
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          add128(acc[i][j], Acc128{(uint64_t)s64[i][j], (uint64_t)(s64[i][j] >> 63)});
    } else {
#pragma unroll 8
      for (int kk = 0; kk < LW_K; ++kk) {
        const int64_t x0 = xs[kk][2 * ty], x1 = xs[kk][2 * ty + 1];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int64_t b = ws[kk][tx + 16 * j];
          mac128(acc[0][j], x0, b);
          mac128(acc[1][j], x1, b);
        }
      }
    }
    __syncthreads();
  }
}

// A 32 x 64 output tile over the K range of blockIdx.z; 16 x 16 threads, 2 x 4 outputs each:
// rows 2 ty, 2 ty + 1 and columns tx + 16 j, so that 16 threads read 16 consecutive staged
// weights (no shared-memory bank conflicts) and write 16 consecutive outputs.
// FINAL (one K split): finish the outputs here; else store the exact partial sums.
template <bool FINAL>
__global__ void __launch_bounds__(256, 2) linear_witness_kernel(const LwArgs a) {
  // staged operands as int64 and as doubles (exact below 2^53), and per stage parity the ORs of
  // |x| and |w|: LW_SMEM bytes of dynamic shared memory
  extern __shared__ __align__(16) unsigned char lw_smem[];
  auto xs = (int64_t(*)[LW_TM + 1])lw_smem;
  auto ws = (int64_t(*)[LW_TN + 1])(lw_smem + LW_XS_BYTES);
  auto xd = (double(*)[LW_TM + 1])(lw_smem + LW_XS_BYTES + LW_WS_BYTES);
  auto wd = (double(*)[LW_TN + 1])(lw_smem + 2 * LW_XS_BYTES + LW_WS_BYTES);
  auto mags = (unsigned long long(*)[2])(lw_smem + 2 * (LW_XS_BYTES + LW_WS_BYTES));
  const unsigned tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const size_t r0 = (size_t)blockIdx.y * LW_TM, c0 = (size_t)blockIdx.x * LW_TN;
  const size_t kb = (size_t)blockIdx.z * a.kchunk, ke = min(a.inner, kb + a.kchunk);
  Acc128 acc[2][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = Acc128{0, 0};
  if (threadIdx.x == 0) mags[0][0] = mags[0][1] = mags[1][0] = mags[1][1] = 0;
  __syncthreads();
  lw_tile_loop(a, xs, ws, xd, wd, mags, r0, c0, kb, ke, acc);
  bool bad = false;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const size_t r = r0 + 2 * ty + i, c = c0 + tx + 16 * j;
      if (r >= a.rows || c >= a.cols) continue;
      const size_t o = r * a.cols + c;
      if (FINAL)
        bad |= !lw_finish(acc[i][j], a.bias, c, a.d, o, a.q, a.rem, a.y, a.yf);
      else
        a.part[(size_t)blockIdx.z * a.rows * a.cols + o] = acc[i][j];
    }
  if (bad) atomicOr(a.err, 1);
}

// Sums the K splits of every output (exactly) and finishes it.
__global__ void linear_witness_finish_kernel(const LwArgs a, unsigned nsplit) {
  const size_t n = a.rows * a.cols;
  bool bad = false;
  for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < n;
       o += (size_t)gridDim.x * blockDim.x) {
    Acc128 s{0, 0};
    for (unsigned z = 0; z < nsplit; ++z) add128(s, a.part[(size_t)z * n + o]);
    bad |= !lw_finish(s, a.bias, o % a.cols, a.d, o, a.q, a.rem, a.y, a.yf);
  }
  if (bad) atomicOr(a.err, 1);
}

// layer_norm (proofsys/src/model.rs:241-279), one CTA per row: exact 128-bit sums of x and x^2,
// vs = d sx2 - sx^2, std = round_sqrt(vs + 1) (the double square root rounded half away from zero,
// tensor.rs:218-222; sqrt is correctly rounded on both sides), then per entry dividend =
// gain (d x - sx), quotient = floor(dividend / std), output = quotient + bias.
struct LnArgs {
  const int64_t *x, *gain, *bias;
  size_t rows, d;
  int64_t *sum_x, *sum_x2, *var_sum, *stdv, *dividend, *quotient, *output;
  int* err;
};
__device__ __forceinline__ __int128 as128(const Acc128& a) {
  return (__int128)(((unsigned __int128)a.hi << 64) | a.lo);
}
__device__ __forceinline__ bool fits64(__int128 v) {
  return v >= (__int128)INT64_MIN && v <= (__int128)INT64_MAX;
}
__global__ void __launch_bounds__(256) layer_norm_witness_kernel(const LnArgs a) {
  __shared__ Acc128 red[2][256];
  __shared__ int64_t s_sx, s_st;
  __shared__ int s_ok;
  const size_t r = blockIdx.x, d = a.d;
  const int64_t* xr = a.x + r * d;
  Acc128 s1{0, 0}, s2{0, 0};
  for (size_t c = threadIdx.x; c < d; c += blockDim.x) {
    const int64_t v = xr[c];
    add128(s1, Acc128{(uint64_t)v, (uint64_t)(v >> 63)});
    mac128(s2, v, v);
  }
  red[0][threadIdx.x] = s1;
  red[1][threadIdx.x] = s2;
  __syncthreads();
  for (unsigned h = blockDim.x / 2; h; h >>= 1) {
    if (threadIdx.x < h) {
      add128(red[0][threadIdx.x], red[0][threadIdx.x + h]);
      add128(red[1][threadIdx.x], red[1][threadIdx.x + h]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const __int128 sx = as128(red[0][0]), sx2 = as128(red[1][0]);
    const __int128 vs = sx2 * (__int128)d - sx * sx;
    int ok = fits64(sx) && fits64(sx2) && fits64(vs) && vs >= 0;
    int64_t st = 1;
    if (ok) {
      const double root = sqrt((double)(unsigned long long)((uint64_t)(int64_t)vs + 1));
      st = (int64_t)llround(root);
      a.sum_x[r] = (int64_t)sx;
      a.sum_x2[r] = (int64_t)sx2;
      a.var_sum[r] = (int64_t)vs;
      a.stdv[r] = st;
    }
    s_sx = ok ? (int64_t)sx : 0;
    s_st = st;
    s_ok = ok;
  }
  __syncthreads();
  if (!s_ok) {
    if (threadIdx.x == 0) atomicOr(a.err, 1);
    return;
  }
  const int64_t sx = s_sx, st = s_st;
  bool bad = false;
  for (size_t c = threadIdx.x; c < d; c += blockDim.x) {
    const __int128 av = (__int128)a.gain[c] * ((__int128)d * (__int128)xr[c] - (__int128)sx);
    if (!fits64(av)) {  // the reference's checked dividend
      bad = true;
      continue;
    }
    const int64_t v = (int64_t)av;
    int64_t q = v / st;
    if (v % st < 0) q -= 1;
    const size_t o = r * d + c;
    a.dividend[o] = v;
    a.quotient[o] = q;
    a.output[o] = (int64_t)((uint64_t)q + (uint64_t)a.bias[c]);
  }
  if (bad) atomicOr(a.err, 1);
}

}  // namespace

void linear_witness_dev(lgs_ctx* c, const int64_t* x, size_t rows, size_t inner, const int64_t* w,
                        size_t cols, bool w_transposed, const int64_t* bias, int64_t divisor,
                        bool on_device, int64_t* q, int64_t* rem, int64_t* y, uint64_t* y_field) {
  if (divisor <= 0) throw ShapeError("linear witness: the divisor must be positive");
  if (rows == 0 || inner == 0 || cols == 0) throw ShapeError("linear witness: empty matrix");
  if (rows > ((size_t)1 << 20) || cols > ((size_t)1 << 24) || inner > ((size_t)1 << 24))
    throw ShapeError("linear witness: matrix too large");
  cudaStream_t st = c->st;
  Arena& ar = c->arena;
  ar.begin();
  const size_t nx = rows * inner, nw = inner * cols, no = rows * cols;
  auto in = [&](const int64_t* h, size_t n) -> const int64_t* {
    if (!h) return nullptr;
    if (on_device) return h;
    int64_t* d = ar.get<int64_t>(n);
    h2d_staged(c, d, h, n * 8, st);
    return d;
  };
  const int64_t* dx = in(x, nx);
  const int64_t* dw = in(w, nw);
  const int64_t* db = in(bias, cols);
  int64_t *dq = q, *dr = rem, *dy = y;
  uint64_t* df = y_field;
  if (!on_device) {
    dq = ar.get<int64_t>(no);
    dr = ar.get<int64_t>(no);
    dy = ar.get<int64_t>(no);
    df = y_field ? ar.get<uint64_t>(no) : nullptr;
  }
  int* derr = ar.get<int>(2);  // error word, then the tensor path's operand-range flag
  LGS_CUDA(cudaMemsetAsync(derr, 0, 2 * sizeof(int), st));
  int herr = 0;
  bool done = false;
  if (c->witness_path == 0) {
    // operands within the limb encodings (every integer GPT-2 layer): the tensor cores
    linear_witness_tc(c, dx, rows, inner, dw, cols, w_transposed, db, divisor, dq, dr, dy, df,
                      derr, derr + 1);
    int flags[2] = {0, 0};
    LGS_CUDA(cudaMemcpyAsync(flags, derr, sizeof(flags), cudaMemcpyDeviceToHost, st));
    LGS_CUDA(cudaStreamSynchronize(st));
    if (flags[0] >= 16)
      throw DeviceTimeout("linear witness: a bounded device wait gave up (code " +
                          std::to_string(flags[0]) + ")");
    done = flags[1] == 0;  // else an operand needs more than its limbs: the CUDA-core kernel
    if (done) herr = flags[0];
    else LGS_CUDA(cudaMemsetAsync(derr, 0, 2 * sizeof(int), st));
  }
  if (!done) {
  // Few rows (GPT-2 runs 31 positions) leave most SMs idle: split K until there are about two
  // CTAs per SM, each with at least 128 values of K, and sum the exact partials afterwards.
  const size_t tiles = ((cols + LW_TN - 1) / LW_TN) * ((rows + LW_TM - 1) / LW_TM);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  size_t split = std::max<size_t>(1, (2 * (size_t)nsm + tiles - 1) / tiles);
  split = std::min<size_t>(split, std::max<size_t>(1, inner / 128));
  split = std::min<size_t>(split, 64);
  size_t kchunk = (inner + split - 1) / split;
  kchunk = (kchunk + LW_K - 1) / LW_K * LW_K;
  split = (inner + kchunk - 1) / kchunk;
  LwArgs a{dx, dw, db, rows, inner, cols, kchunk, divisor, w_transposed ? 1 : 0, nullptr,
           dq, dr, dy, df, derr};
  const dim3 grid((unsigned)((cols + LW_TN - 1) / LW_TN), (unsigned)((rows + LW_TM - 1) / LW_TM),
                  (unsigned)split);
  LGS_CUDA(cudaFuncSetAttribute(linear_witness_kernel<true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LW_SMEM));
  LGS_CUDA(cudaFuncSetAttribute(linear_witness_kernel<false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LW_SMEM));
  StageTimer t(c->prof, st, "linear_witness_cores");
  if (split == 1) {
    linear_witness_kernel<true><<<grid, 256, LW_SMEM, st>>>(a);
    LGS_LAUNCH_CHECK();
  } else {
    a.part = ar.get<Acc128>(split * no);
    linear_witness_kernel<false><<<grid, 256, LW_SMEM, st>>>(a);
    LGS_LAUNCH_CHECK();
    const unsigned blocks = (unsigned)std::min<size_t>((no + 255) / 256, 148 * 8);
    linear_witness_finish_kernel<<<blocks, 256, 0, st>>>(a, (unsigned)split);
    LGS_LAUNCH_CHECK();
  }
  LGS_CUDA(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
  }
  if (!on_device) {
    LGS_CUDA(cudaMemcpyAsync(q, dq, no * 8, cudaMemcpyDeviceToHost, st));
    LGS_CUDA(cudaMemcpyAsync(rem, dr, no * 8, cudaMemcpyDeviceToHost, st));
    LGS_CUDA(cudaMemcpyAsync(y, dy, no * 8, cudaMemcpyDeviceToHost, st));
    if (y_field) LGS_CUDA(cudaMemcpyAsync(y_field, df, no * 8, cudaMemcpyDeviceToHost, st));
  }
  LGS_CUDA(cudaStreamSynchronize(st));
  if (herr) throw ShapeError("linear witness: a product or Q + bias leaves the i64 range");
}

}  // namespace lgs

namespace lgs {

void layer_norm_witness_dev(lgs_ctx* c, const int64_t* x, size_t rows, size_t d,
                            const int64_t* gain, const int64_t* bias, bool on_device,
                            int64_t* const per_row[4], int64_t* const per_entry[3]) {
  if (rows == 0 || d == 0) throw ShapeError("layer norm witness: empty matrix");
  if (rows > ((size_t)1 << 24) || d > ((size_t)1 << 24))
    throw ShapeError("layer norm witness: matrix too large");
  cudaStream_t st = c->st;
  Arena& ar = c->arena;
  ar.begin();
  auto in = [&](const int64_t* h, size_t n) -> const int64_t* {
    if (on_device) return h;
    int64_t* dv = ar.get<int64_t>(n);
    h2d_staged(c, dv, h, n * 8, st);
    return dv;
  };
  int64_t* dr[4];
  int64_t* de[3];
  for (int i = 0; i < 4; ++i) dr[i] = on_device ? per_row[i] : ar.get<int64_t>(rows);
  for (int i = 0; i < 3; ++i) de[i] = on_device ? per_entry[i] : ar.get<int64_t>(rows * d);
  int* derr = ar.get<int>(1);
  LGS_CUDA(cudaMemsetAsync(derr, 0, sizeof(int), st));
  LnArgs a{in(x, rows * d), in(gain, d), in(bias, d), rows, d, dr[0], dr[1], dr[2], dr[3],
           de[0], de[1], de[2], derr};
  layer_norm_witness_kernel<<<(unsigned)rows, 256, 0, st>>>(a);
  LGS_LAUNCH_CHECK();
  int herr = 0;
  LGS_CUDA(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (!on_device) {
    for (int i = 0; i < 4; ++i)
      LGS_CUDA(cudaMemcpyAsync(per_row[i], dr[i], rows * 8, cudaMemcpyDeviceToHost, st));
    for (int i = 0; i < 3; ++i)
      LGS_CUDA(cudaMemcpyAsync(per_entry[i], de[i], rows * d * 8, cudaMemcpyDeviceToHost, st));
  }
  LGS_CUDA(cudaStreamSynchronize(st));
  if (herr) throw ShapeError("layer norm witness: a sum, the variance or a dividend leaves the i64 range");
}

}  // namespace lgs

// ---- softmax and lookup gathers of the integer GPT-2 (proofsys/src/model.rs:362-373, 409-443) ----
namespace lgs {

namespace {

// softmax (model.rs:409-443), causal: for head h and row i, x_max = max_{j <= i} s[i][j],
// exp[i][j] = exp_lut[s[i][j] - x_max + offset] and prob[i][j] = floor(exp[i][j] scale / sum)
// for j <= i (zero above the diagonal), sum_exp = sum_j exp[i][j].  One thread per (head, row).
__global__ void softmax_witness_kernel(const int64_t* __restrict__ s, unsigned heads, unsigned n,
                                       const int64_t* __restrict__ lut, size_t lut_len,
                                       int64_t offset, int64_t scale, int64_t* __restrict__ x_max,
                                       int64_t* __restrict__ ex, int64_t* __restrict__ sum_exp,
                                       int64_t* __restrict__ prob, int* __restrict__ err) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)heads * n) return;
  const size_t i = t % n, base = t * n;  // row i of head t / n: s[base + j]
  int64_t mx = s[base];
  for (size_t j = 1; j <= i; ++j) mx = max(mx, s[base + j]);
  x_max[t] = mx;
  int64_t sum = 0;
  bool bad = false;
  for (size_t j = 0; j < n; ++j) {
    int64_t e = 0;
    if (j <= i) {
      const int64_t idx = s[base + j] - mx + offset;
      if (idx < 0 || (uint64_t)idx >= lut_len) {
        bad = true;
      } else {
        e = lut[idx];
        sum += e;
      }
    }
    ex[base + j] = e;
  }
  sum_exp[t] = sum;
  if (sum <= 0) bad = true;  // the reference's floor_div_i128 asserts a positive divisor
  for (size_t j = 0; j < n; ++j) {
    int64_t p = 0;
    if (j <= i && !bad) {
      const __int128 a = (__int128)ex[base + j] * scale;
      __int128 q = a / sum;
      if (a % sum < 0) q -= 1;
      if (q < (__int128)INT64_MIN || q > (__int128)INT64_MAX) bad = true;
      p = (int64_t)q;
    }
    prob[base + j] = p;
  }
  if (bad) atomicOr(err, 1);
}

// out[i] = lut[v[i] + offset] (the GELU activation, model.rs:362-373).
__global__ void lut_gather_kernel(const int64_t* __restrict__ v, size_t count,
                                  const int64_t* __restrict__ lut, size_t lut_len, int64_t offset,
                                  int64_t* __restrict__ out, int* __restrict__ err) {
  bool bad = false;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x) {
    const int64_t idx = v[i] + offset;
    if (idx < 0 || (uint64_t)idx >= lut_len) {
      bad = true;
      out[i] = 0;
    } else {
      out[i] = lut[idx];
    }
  }
  if (bad) atomicOr(err, 1);
}

// Uploads host arrays (or passes device ones), runs `launch`, reads the outputs back.
template <class F>
void run_small(lgs_ctx* c, bool on_device, std::initializer_list<std::pair<const int64_t*, size_t>> ins,
               std::initializer_list<std::pair<int64_t*, size_t>> outs, const char* what,
               F&& launch) {
  cudaStream_t st = c->st;
  Arena& ar = c->arena;
  ar.begin();
  std::vector<const int64_t*> din;
  for (auto& p : ins) {
    if (on_device) {
      din.push_back(p.first);
    } else {
      int64_t* d = ar.get<int64_t>(p.second);
      h2d_staged(c, d, p.first, p.second * 8, st);
      din.push_back(d);
    }
  }
  std::vector<int64_t*> dout;
  for (auto& p : outs) dout.push_back(on_device ? p.first : ar.get<int64_t>(p.second));
  int* derr = ar.get<int>(1);
  LGS_CUDA(cudaMemsetAsync(derr, 0, sizeof(int), st));
  launch(din, dout, derr);
  int herr = 0;
  LGS_CUDA(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (!on_device) {
    size_t k = 0;
    for (auto& p : outs) {
      LGS_CUDA(cudaMemcpyAsync(p.first, dout[k], p.second * 8, cudaMemcpyDeviceToHost, st));
      ++k;
    }
  }
  LGS_CUDA(cudaStreamSynchronize(st));
  if (herr) throw ShapeError(what);
}

}  // namespace

void softmax_witness_dev(lgs_ctx* c, const int64_t* scores, unsigned heads, unsigned n,
                         const int64_t* lut, size_t lut_len, int64_t offset, int64_t scale,
                         bool on_device, int64_t* x_max, int64_t* ex, int64_t* sum_exp,
                         int64_t* prob) {
  if (heads == 0 || n == 0 || lut_len == 0) throw ShapeError("softmax witness: empty input");
  if ((size_t)heads * n > ((size_t)1 << 24) || n > 65536) throw ShapeError("softmax witness: too large");
  const size_t hn = (size_t)heads * n, hnn = hn * n;
  run_small(c, on_device, {{scores, hnn}, {lut, lut_len}},
            {{x_max, hn}, {ex, hnn}, {sum_exp, hn}, {prob, hnn}},
            "softmax witness: an exp index outside the table, or a zero sum",
            [&](const std::vector<const int64_t*>& in, const std::vector<int64_t*>& out, int* err) {
              softmax_witness_kernel<<<(unsigned)((hn + 127) / 128), 128, 0, c->st>>>(
                  in[0], heads, n, in[1], lut_len, offset, scale, out[0], out[1], out[2], out[3],
                  err);
              LGS_LAUNCH_CHECK();
            });
}

void lut_gather_dev(lgs_ctx* c, const int64_t* v, size_t count, const int64_t* lut,
                    size_t lut_len, int64_t offset, bool on_device, int64_t* out) {
  if (count == 0 || lut_len == 0) throw ShapeError("lookup gather: empty input");
  run_small(c, on_device, {{v, count}, {lut, lut_len}}, {{out, count}},
            "lookup gather: an index outside the table",
            [&](const std::vector<const int64_t*>& in, const std::vector<int64_t*>& o, int* err) {
              const unsigned blocks = (unsigned)std::min<size_t>((count + 255) / 256, 148 * 8);
              lut_gather_kernel<<<blocks, 256, 0, c->st>>>(in[0], count, in[1], lut_len, offset,
                                                           o[0], err);
              LGS_LAUNCH_CHECK();
            });
}

}  // namespace lgs
