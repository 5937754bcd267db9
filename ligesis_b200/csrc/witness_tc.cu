// proofsys' rescaled linear layer (proofsys/src/model.rs:360-374 and the vocabulary head
// :225-228: Q, REM = floor_div(X W, divisor), Y = Q + bias) with the contraction on the int8
// tensor cores (tcgen05.mma.kind::i8), exactly.
//
// The integer GPT-2's activations are fixed-point values of about 21 bits and its weights fit in
// 16 bits, so the product splits into byte limbs with offset-binary encodings:
//   x' = x + 2^23 in [0, 2^24): three unsigned limbs x'_0..2;  w' = w + 2^15 in [0, 2^16): two.
// Every limb product u8 x u8 sums exactly in int32 (groups of at most two limb pairs per shift,
// at most 16384 values of K per CTA), and
//   sum_k x w = sum_g 2^(8g) S_g - 2^15 sum_k x' - 2^23 sum_k w' + K 2^38,
//   S_g = sum over limb pairs i + j = g of sum_k x'_i w'_j.
// sum_k w' comes out of the tensor cores too: the row after the last x row of a tile is all ones
// in limb 0.  sum_k x' is summed by the threads that stage x.  A value outside those ranges sets
// a flag and the caller runs the CUDA-core kernel instead (witness.cu), which handles any i64.
//
// One CTA computes a 128-column x NR-row output tile (D^T = W_tile X^T: M = 128 output columns,
// N = NR <= 64 rows) over a K range, in chunks of 128 values of K:
//   warps 0-7  load W and X from global memory, convert them to limbs in the 128-byte swizzled
//              K-major tiles of a 2-stage pipeline (the weights are read from HBM exactly once)
//   warp 0     also allocates the TMEM and, once all warps have staged a chunk, one of its
//              threads issues the chunk's MMAs (M128 N=NR K32, 6 limb pairs, 4 K steps) into
//              four accumulators of NR columns
//   warps 0-3  afterwards: drain the accumulators, recombine, finish the outputs.
// When K is split over CTAs (to fill the GPU), each split adds its exact int64 sum into a zeroed
// buffer and the last CTA of a tile (a counter per tile) finishes it.  Every wait is bounded.
#include "prover.cuh"
#include "tcgen05.cuh"
#include "witness.cuh"

namespace lgs {

namespace {

constexpr int WT_M = 128;        // output columns per tile (MMA M)
constexpr int WT_KC = 128;       // K values per chunk (one 128-byte row of a limb tile)
constexpr int WT_LX = 3, WT_LW = 2, WT_NG = WT_LX + WT_LW - 1;
constexpr int WT_STAGES = 2;
constexpr int WT_PROD = 256;     // producer threads (warps 0-7)
constexpr int WT_THREADS = WT_PROD;
constexpr int WT_NR_MAX = 64;
constexpr int64_t WT_OX = (int64_t)1 << 23, WT_OW = (int64_t)1 << 15;
constexpr size_t WT_A_TILE = (size_t)WT_M * WT_KC;  // bytes of one W limb tile
constexpr size_t WT_KMAX = 16384;  // K values per CTA that keep every S_g within int32

__host__ __device__ constexpr size_t wt_stage_bytes(unsigned nr) {
  return WT_LW * WT_A_TILE + (size_t)WT_LX * nr * WT_KC;
}
size_t wt_smem_bytes(unsigned nr) {
  return WT_STAGES * wt_stage_bytes(nr) + 1024 /*align*/ + WT_NR_MAX * 8 /*sum x'*/ + 128;
}

struct WtArgs {
  const int64_t* x;   // rows x inner
  const int64_t* w;   // cols x inner (wt) or inner x cols
  const int64_t* bias;
  size_t rows, inner, cols, kchunk;
  unsigned nsplit, nr, nrv;  // MMA N, and the x rows of a row tile (nrv < nr: one ones row)
  int wt;
  int64_t d;
  int64_t *q, *rem, *y;
  uint64_t* yf;
  unsigned long long* acc;  // rows x cols, zeroed (nsplit > 1)
  unsigned* count;          // per tile, zeroed (nsplit > 1)
  int* err;                 // 1: a result leaves the i64 range; >= 16: a bounded wait gave up
  int* range;               // an operand outside the limb encodings
  long long budget;
  const uint8_t* xl;        // the X limb tiles of every (row tile, chunk), x_limbs_kernel
  const uint32_t* xsum;     // sum of x' per (row tile, chunk, row)
  size_t chunks;            // chunks of 128 values of K in the whole inner dimension
};

// w' = w + 2^15 of a value in range, 0 for padding (outside the matrix); flags a value that
// does not fit 16 bits.
__device__ __forceinline__ uint32_t w_enc(int64_t v, bool valid, bool& bad) {
  const uint64_t e = (uint64_t)v + (uint64_t)WT_OW;
  bad |= valid && (e >> 16) != 0;
  return valid ? (uint32_t)(e & 0xFFFFu) : 0u;
}
// x' = x + 2^23 likewise (24 bits).
__device__ __forceinline__ uint32_t x_enc(int64_t v, bool valid, bool& bad) {
  const uint64_t e = (uint64_t)v + (uint64_t)WT_OX;
  bad |= valid && (e >> 24) != 0;
  return valid ? (uint32_t)(e & 0xFFFFFFu) : 0u;
}
// Byte l of two encoded values as a 16-bit pair (value a in the low byte).
__device__ __forceinline__ uint32_t pair_byte(uint32_t a, uint32_t b, int l) {
  return ((a >> (8 * l)) & 255u) | (((b >> (8 * l)) & 255u) << 8);
}

// A row of a 128-byte limb tile from one warp: lane t holds the encoded values of K offsets
// 2t, 2t + 1 (ea, eb) and 64 + 2t, 64 + 2t + 1 (ec, ed).  Lane pairs swap halves so that each
// lane owns four consecutive K offsets (even lanes 4j.., odd lanes 64 + 4j..) and stores one
// 32-bit word per limb.  L limbs (2 or 3).
template <int L>
__device__ __forceinline__ void store_row(uint8_t* const (&tiles)[L], uint32_t row,
                                          uint32_t ea, uint32_t eb, uint32_t ec, uint32_t ed) {
  const unsigned lane = threadIdx.x & 31;
  const bool odd = lane & 1;
  const uint32_t kb = odd ? 62 + 2 * lane : 2 * lane;
#pragma unroll
  for (int l = 0; l < L; ++l) {
    const uint32_t mine_lo = pair_byte(ea, eb, l), mine_hi = pair_byte(ec, ed, l);
    const uint32_t other = __shfl_xor_sync(0xffffffffu, odd ? mine_lo : mine_hi, 1);
    const uint32_t word = odd ? (other | (mine_hi << 16)) : (mine_lo | (other << 16));
    *(uint32_t*)(tiles[l] + tc::sw128_off(row, kb)) = word;
  }
}

__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Group q (steps 2q, 2q + 1 of 16) of the W values this thread stages for the chunk at k0:
//   w transposed (W[c][k]): step s is output column m = 8 s + warp, the values at K offsets
//     2 lane, 2 lane + 1, 64 + 2 lane, 64 + 2 lane + 1 (two 16-byte loads when vec);
//   else (W[k][c]): column m = 32 (warp % 4) + lane, K offsets 8 s + 4 (warp / 4) + 0..3.
// Every address is clamped into the matrix (no branch, so the loads issue back to back);
// store_w_group zeroes the values outside it.
template <bool WT, bool VEC>
__device__ __forceinline__ void load_w_group(const WtArgs& a, size_t c0, size_t k0, size_t ke,
                                             unsigned warp, unsigned lane, int q,
                                             int64_t (&v)[8]) {
  if constexpr (WT) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const size_t c = min(c0 + 8 * (2 * q + i) + warp, a.cols - 1);
      const int64_t* p = a.w + c * a.inner;
      const size_t ka = k0 + 2 * lane, kb2 = k0 + 64 + 2 * lane;
      if constexpr (VEC) {  // inner even: ke - 2 >= k0 is even: both 16-byte loads stay in the row
        const longlong2 x = __ldg((const longlong2*)(p + min(ka, ke - 2)));
        const longlong2 y = __ldg((const longlong2*)(p + min(kb2, ke - 2)));
        v[4 * i] = x.x, v[4 * i + 1] = x.y, v[4 * i + 2] = y.x, v[4 * i + 3] = y.y;
      } else {
        v[4 * i] = __ldg(p + min(ka, ke - 1));
        v[4 * i + 1] = __ldg(p + min(ka + 1, ke - 1));
        v[4 * i + 2] = __ldg(p + min(kb2, ke - 1));
        v[4 * i + 3] = __ldg(p + min(kb2 + 1, ke - 1));
      }
    }
  } else {
    const size_t c = min(c0 + 32 * (warp & 3) + lane, a.cols - 1);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const size_t kk = k0 + 8 * (2 * q + i) + 4 * (warp >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j) v[4 * i + j] = __ldg(a.w + min(kk + j, ke - 1) * a.cols + c);
    }
  }
}
template <bool WT>
__device__ __forceinline__ void store_w_group(const WtArgs& a, uint8_t* const (&tiles)[WT_LW],
                                              size_t c0, size_t k0, size_t ke, unsigned warp,
                                              unsigned lane, int q, const int64_t (&v)[8],
                                              bool& bad) {
  if constexpr (WT) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const unsigned m = 8 * (2 * q + i) + warp;
      const bool ok = c0 + m < a.cols;
      const size_t ka = k0 + 2 * lane, kb2 = k0 + 64 + 2 * lane;
      const uint32_t e0 = w_enc(v[4 * i], ok && ka < ke, bad);
      const uint32_t e1 = w_enc(v[4 * i + 1], ok && ka + 1 < ke, bad);
      const uint32_t e2 = w_enc(v[4 * i + 2], ok && kb2 < ke, bad);
      const uint32_t e3 = w_enc(v[4 * i + 3], ok && kb2 + 1 < ke, bad);
      store_row<WT_LW>(tiles, m, e0, e1, e2, e3);
    }
  } else {
    const unsigned m = 32 * (warp & 3) + lane;
    const bool ok = c0 + m < a.cols;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const unsigned kk = 8 * (2 * q + i) + 4 * (warp >> 2);
      uint32_t w0 = 0, w1 = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint32_t e = w_enc(v[4 * i + j], ok && k0 + kk + j < ke, bad);
        w0 |= (e & 255u) << (8 * j);
        w1 |= ((e >> 8) & 255u) << (8 * j);
      }
      *(uint32_t*)(tiles[0] + tc::sw128_off(m, kk)) = w0;
      *(uint32_t*)(tiles[1] + tc::sw128_off(m, kk)) = w1;
    }
  }
}

// The X side of every chunk, once per launch: for row tile blockIdx.y and the chunk of K values
// [128 blockIdx.x, 128 blockIdx.x + 128), the three limb tiles exactly as the main kernel's
// shared memory holds them (rows below nrv data, row nrv all ones in limb 0, the rest zero), and
// each data row's sum of x' over the chunk.  A value outside 24 bits sets *range.
__global__ void __launch_bounds__(256) x_limbs_kernel(const WtArgs a, uint8_t* __restrict__ xl,
                                                      uint32_t* __restrict__ xsum) {
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nr = a.nr;
  const size_t chunks = gridDim.x, chunk = blockIdx.x, tile = blockIdx.y;
  const size_t r0 = tile * a.nrv, k0 = chunk * WT_KC;
  uint8_t* base = xl + (tile * chunks + chunk) * (size_t)(WT_LX * nr * WT_KC);
  uint8_t* const tiles[WT_LX] = {base, base + nr * WT_KC, base + 2 * nr * WT_KC};
  bool bad = false;
  for (unsigned r = warp; r < nr; r += 8) {
    const size_t gr = r0 + r;
    const bool data = r < a.nrv && gr < a.rows;
    uint32_t e[4] = {0, 0, 0, 0};
    if (data) {
      const int64_t* p = a.x + gr * a.inner;
      const size_t ks[4] = {k0 + 2 * lane, k0 + 2 * lane + 1, k0 + 64 + 2 * lane,
                            k0 + 64 + 2 * lane + 1};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const bool valid = ks[i] < a.inner;
        e[i] = x_enc(valid ? __ldg(p + ks[i]) : 0, valid, bad);
      }
      const unsigned part = __reduce_add_sync(0xffffffffu, e[0] + e[1] + e[2] + e[3]);
      if (lane == 0) xsum[(tile * chunks + chunk) * nr + r] = part;
    } else {
      if (r == a.nrv) e[0] = e[1] = e[2] = e[3] = 1;
      if (lane == 0) xsum[(tile * chunks + chunk) * nr + r] = 0;
    }
    store_row<WT_LX>(tiles, r, e[0], e[1], e[2], e[3]);
  }
  if (bad) atomicExch(a.range, 1);
}

// WT: W is cols x inner (else inner x cols); VEC: W rows start 16-byte aligned (16-byte loads).
template <bool WT, bool VEC>
__global__ void __launch_bounds__(WT_THREADS, 2) linear_witness_tc_kernel(const WtArgs a) {
  extern __shared__ uint8_t wt_smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)wt_smem_raw + 1023) & ~(uintptr_t)1023);
  const unsigned nr = a.nr;
  const size_t stage_bytes = wt_stage_bytes(nr);
  unsigned long long* sx = (unsigned long long*)(smem + WT_STAGES * stage_bytes);
  uint64_t* bars = (uint64_t*)(sx + WT_NR_MAX);
  uint32_t* tmem_holder = (uint32_t*)(bars + 3 * WT_STAGES + 2);
  const uint32_t full0 = tc::smem_u32(&bars[0]), empty0 = tc::smem_u32(&bars[WT_STAGES]);
  const uint32_t xbar0 = tc::smem_u32(&bars[2 * WT_STAGES]);  // the X tiles' bulk copies
  const uint32_t accf = tc::smem_u32(&bars[3 * WT_STAGES]);
  const uint32_t drain = tc::smem_u32(&bars[3 * WT_STAGES + 1]);
  __shared__ volatile int s_fail;
  __shared__ int s_last;
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t c0 = (size_t)blockIdx.x * WT_M, r0 = (size_t)blockIdx.y * a.nrv;
  const size_t kb = (size_t)blockIdx.z * a.kchunk, ke = min(a.inner, kb + a.kchunk);
  const unsigned nchunks = (unsigned)((ke - kb + WT_KC - 1) / WT_KC);
  const unsigned tcols = nr * WT_NG <= 64 ? 64 : (nr * WT_NG <= 128 ? 128 : 256);

  if (tid == 0) {
    s_fail = 0;
    for (int s = 0; s < WT_STAGES; ++s) {
      tc::mbar_init(full0 + 8 * s, WT_PROD);
      tc::mbar_init(empty0 + 8 * s, 1);
      tc::mbar_init(xbar0 + 8 * s, 1);
    }
    tc::mbar_init(accf, 1);
    tc::mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(tmem_holder)),
                 "r"(tcols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_holder;
  unsigned x_issued = 0;  // thread 0: X tile copies issued

  {
    // ---- producers: the W tile (128 output columns) of each chunk as limbs, in eight groups of
    // eight values per thread; the loads run three groups ahead of the stores (a ring of four
    // register buffers, across chunk boundaries).  Thread 0 also fetches the chunk's X limb
    // tiles (made once per launch by x_limbs_kernel) with one bulk copy.
    bool bad = false;
    const size_t xt_bytes = (size_t)WT_LX * nr * WT_KC;
    int64_t b0[8], b1[8], b2[8], b3[8];
    load_w_group<WT, VEC>(a, c0, kb, ke, warp, lane, 0, b0);
    load_w_group<WT, VEC>(a, c0, kb, ke, warp, lane, 1, b1);
    load_w_group<WT, VEC>(a, c0, kb, ke, warp, lane, 2, b2);
    for (unsigned t = 0; t < nchunks; ++t) {
      const unsigned s = t % WT_STAGES;
      const size_t k0 = kb + (size_t)t * WT_KC, k1 = k0 + WT_KC;
      const bool more = t + 1 < nchunks;
      if (t >= WT_STAGES) {  // one lane waits, so the warp decides as one (it shuffles below)
        bool ok = true;
        if (lane == 0) ok = tc::mbar_wait(empty0 + 8 * s, ((t / WT_STAGES) - 1) & 1, &s_fail,
                                          a.budget);
        if (!__shfl_sync(0xffffffffu, ok, 0)) {
          if (lane == 0 && !s_fail) tc::flag_failure(&s_fail, a.err, 18);
          break;
        }
      }
      uint8_t* st = smem + s * stage_bytes;
      uint8_t* const wt_tiles[WT_LW] = {st, st + WT_A_TILE};
      if (tid == 0) {
        const uint32_t bar = xbar0 + 8 * s;
        tc::mbar_arrive_tx(bar, (uint32_t)xt_bytes);
        x_issued = t + 1;
        const uint8_t* src = a.xl + (blockIdx.y * a.chunks + kb / WT_KC + t) * xt_bytes;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(tc::smem_u32(st + WT_LW * WT_A_TILE)),
            "l"(src), "r"((uint32_t)xt_bytes), "r"(bar)
            : "memory");
      }
      load_w_group<WT, VEC>(a, c0, k0, ke, warp, lane, 3, b3);
      store_w_group<WT>(a, wt_tiles, c0, k0, ke, warp, lane, 0, b0, bad);
      load_w_group<WT, VEC>(a, c0, k0, ke, warp, lane, 4, b0);
      store_w_group<WT>(a, wt_tiles, c0, k0, ke, warp, lane, 1, b1, bad);
      load_w_group<WT, VEC>(a, c0, k0, ke, warp, lane, 5, b1);
      store_w_group<WT>(a, wt_tiles, c0, k0, ke, warp, lane, 2, b2, bad);
      load_w_group<WT, VEC>(a, c0, k0, ke, warp, lane, 6, b2);
      store_w_group<WT>(a, wt_tiles, c0, k0, ke, warp, lane, 3, b3, bad);
      load_w_group<WT, VEC>(a, c0, k0, ke, warp, lane, 7, b3);
      store_w_group<WT>(a, wt_tiles, c0, k0, ke, warp, lane, 4, b0, bad);
      if (more) load_w_group<WT, VEC>(a, c0, k1, ke, warp, lane, 0, b0);
      store_w_group<WT>(a, wt_tiles, c0, k0, ke, warp, lane, 5, b1, bad);
      if (more) load_w_group<WT, VEC>(a, c0, k1, ke, warp, lane, 1, b1);
      store_w_group<WT>(a, wt_tiles, c0, k0, ke, warp, lane, 6, b2, bad);
      if (more) load_w_group<WT, VEC>(a, c0, k1, ke, warp, lane, 2, b2);
      store_w_group<WT>(a, wt_tiles, c0, k0, ke, warp, lane, 7, b3, bad);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tc::mbar_arrive(full0 + 8 * s);
      if (warp == 0) {
        // MMA issue: once every producer has staged the chunk, 4 K steps x 6 limb pairs, pair
        // (i, j) into accumulator i + j; the commit frees the stage
        bool ok = true;
        if (lane == 0)
          ok = tc::mbar_wait(full0 + 8 * s, (t / WT_STAGES) & 1, &s_fail, a.budget) &&
               tc::mbar_wait(xbar0 + 8 * s, (t / WT_STAGES) & 1, &s_fail, a.budget);
        if (!__shfl_sync(0xffffffffu, ok, 0)) {
          if (lane == 0 && !s_fail) tc::flag_failure(&s_fail, a.err, 16);
          break;
        }
        if (lane == 0) {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t idesc = tc::idesc_u8(WT_M, nr);
          const uint32_t sa = tc::smem_u32(st);
          const uint32_t sb = sa + (uint32_t)(WT_LW * WT_A_TILE);
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
#pragma unroll
            for (int i = 0; i < WT_LX; ++i)
#pragma unroll
              for (int j = 0; j < WT_LW; ++j) {
                // the first pair of each accumulator in the first K step overwrites it
                const bool first = t == 0 && ks == 0 && (j == 1 || i == 0);
                tc::mma_i8(tmem + (uint32_t)((i + j) * nr),
                           tc::sw128_desc(sa + (uint32_t)(j * WT_A_TILE) + 32 * ks),
                           tc::sw128_desc(sb + (uint32_t)(i * nr * WT_KC) + 32 * ks), idesc,
                           first ? 0u : 1u);
              }
          tc::mma_commit(empty0 + 8 * s);
          if (t + 1 == nchunks) tc::mma_commit(accf);
        }
        __syncwarp();
      }
    }
    if (bad) atomicExch(a.range, 1);
    // this CTA's sums of x' per row, from the per-chunk sums
    if (tid < nr) {
      unsigned long long sum = 0;
      for (unsigned t = 0; t < nchunks; ++t)
        sum += a.xsum[(blockIdx.y * a.chunks + kb / WT_KC + t) * nr + tid];
      sx[tid] = sum;
    }
    asm volatile("bar.sync 2, 256;" ::: "memory");
    if (warp < 4) {
      // ---- epilogue (warps 0-3; TMEM lanes 32 warp .. 32 warp + 31 = output columns)
      const bool got = tc::mbar_wait(accf, 0, &s_fail, a.budget);
      uint32_t all;
      asm volatile(
          "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, 1, 128, p;\n"
          " selp.u32 %0, 1, 0, q;\n}\n"
          : "=r"(all)
          : "r"((uint32_t)got)
          : "memory");
      if (!all) {
        if (!s_fail) tc::flag_failure(&s_fail, a.err, 19);
      } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t lane_off = (uint32_t)(32 * warp) << 16;
        const unsigned m = 32 * warp + lane;
        const size_t c = c0 + m;
        const bool col_ok = c < a.cols;
        // sum_k w' of this column: the ones row's entry of each accumulator
        int64_t sw = 0;
        {
          const unsigned blk = a.nrv & ~15u, e = a.nrv & 15u;
#pragma unroll
          for (int g = 0; g < WT_NG; ++g) {
            uint32_t v[16];
            tc::tmem_ld16(tmem + lane_off + (uint32_t)(g * nr) + blk, v);
            tc::tmem_wait_ld();
            uint32_t pick = 0;
#pragma unroll
            for (int i = 0; i < 16; ++i) pick = (unsigned)i == e ? v[i] : pick;
            sw += (int64_t)pick << (8 * g);
          }
        }
        const int64_t kv = (int64_t)(ke - kb);
        const int64_t base = kv * WT_OX * WT_OW - WT_OX * sw;
        bool over = false;
        for (unsigned blk = 0; blk < a.nrv; blk += 16) {
          int64_t pv[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) pv[i] = 0;
#pragma unroll
          for (int g = 0; g < WT_NG; ++g) {
            uint32_t v[16];
            tc::tmem_ld16(tmem + lane_off + (uint32_t)(g * nr) + blk, v);
            tc::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) pv[i] += (int64_t)v[i] << (8 * g);
          }
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const unsigned r = blk + i;
            const size_t gr = r0 + r;
            if (r >= a.nrv || gr >= a.rows || !col_ok) continue;
            const int64_t val = pv[i] - WT_OW * (int64_t)sx[r] + base;
            const size_t o = gr * a.cols + c;
            if (a.nsplit == 1)
              over |= !lw_finish(Acc128{(uint64_t)val, (uint64_t)(val >> 63)}, a.bias, c, a.d, o,
                                 a.q, a.rem, a.y, a.yf);
            else
              atomicAdd(a.acc + o, (unsigned long long)val);
          }
        }
        if (a.nsplit > 1) {
          // the last split of this tile to arrive finishes it from the summed buffer
          __threadfence();
          epi_bar();
          if (tid == 0) {
            const unsigned tile = blockIdx.y * gridDim.x + blockIdx.x;
            s_last = atomicAdd(a.count + tile, 1u) == a.nsplit - 1;
          }
          epi_bar();
          if (s_last) {
            __threadfence();
            for (unsigned r = 0; r < a.nrv; ++r) {
              const size_t gr = r0 + r;
              if (gr >= a.rows || !col_ok) continue;
              const size_t o = gr * a.cols + c;
              const int64_t val = (int64_t)__ldcg(a.acc + o);
              over |= !lw_finish(Acc128{(uint64_t)val, (uint64_t)(val >> 63)}, a.bias, c, a.d,
                                 o, a.q, a.rem, a.y, a.yf);
            }
          }
        }
        if (over) atomicOr(a.err, 1);
      }
    }
  }
  if (tid == 0) {
    // only the newest copy of each stage can still be in flight (an older one was consumed
    // before its stage was refilled): wait for those before the CTA may exit
    for (unsigned g = x_issued > WT_STAGES ? x_issued - WT_STAGES : 0; g < x_issued; ++g)
      if (!tc::mbar_wait_drain(xbar0 + 8 * (g % WT_STAGES), (g / WT_STAGES) & 1))
        atomicExch(a.err, 20);
    // every MMA issued so far has completed once this arrives: wait before the TMEM is freed
    tc::mma_commit(drain);
    if (!tc::mbar_wait_drain(drain, 0)) atomicExch(a.err, 17);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols)
                 : "memory");
  }
}

}  // namespace

void linear_witness_tc(lgs_ctx* c, const int64_t* dx, size_t rows, size_t inner,
                       const int64_t* dw, size_t cols, bool w_transposed, const int64_t* db,
                       int64_t divisor, int64_t* dq, int64_t* dr, int64_t* dy, uint64_t* df,
                       int* derr, int* drange) {
  cudaStream_t st = c->st;
  // row tiles of at most 63 x rows (plus the ones row), balanced
  const size_t ntr = (rows + WT_NR_MAX - 2) / (WT_NR_MAX - 1);
  const unsigned nrv = (unsigned)((rows + ntr - 1) / ntr);
  const unsigned nr = (nrv + 1 + 15) / 16 * 16;
  const size_t smem = wt_smem_bytes(nr);
  const bool vec = w_transposed && (inner % 2 == 0) && (((uintptr_t)dw & 15) == 0);
  auto k = w_transposed ? (vec ? linear_witness_tc_kernel<true, true>
                               : linear_witness_tc_kernel<true, false>)
                        : linear_witness_tc_kernel<false, false>;
  LGS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // two CTAs per SM need the largest shared-memory carveout
  LGS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared));
  // resident CTAs per SM: the launch bounds cap registers for two; shared memory decides
  int nsm = 148, smem_sm = 0;
  LGS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
  LGS_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                                  c->device));
  const size_t per_sm = 2 * (smem + 1024) <= (size_t)smem_sm ? 2 : 1;
  const size_t slots = per_sm * nsm;
  const size_t mt = (cols + WT_M - 1) / WT_M, tiles = mt * ntr;
  const size_t chunks = (inner + WT_KC - 1) / WT_KC;
  // K splits: the fewest that minimise (waves of CTAs) x (chunks per CTA + the fixed cost of a
  // CTA, about three chunks with the split epilogue's atomics and finish), and enough that no
  // CTA sums more than WT_KMAX values of K
  const size_t min_split = (inner + WT_KMAX - 1) / WT_KMAX;
  size_t split = min_split, best = SIZE_MAX;
  for (size_t sp = min_split; sp <= std::min<size_t>(chunks, 64); ++sp) {
    const size_t per = (chunks + sp - 1) / sp;
    const size_t cost = ((tiles * sp + slots - 1) / slots) * (per + 3);
    if (cost < best) best = cost, split = sp;
  }
  const size_t kchunk = (chunks + split - 1) / split * WT_KC;
  split = (inner + kchunk - 1) / kchunk;
  Arena& ar = c->arena;
  WtArgs a{dx, dw, db, rows, inner, cols, kchunk, (unsigned)split, nr, nrv,
           w_transposed ? 1 : 0, divisor, dq, dr, dy, df, nullptr, nullptr, derr, drange, 0};
  a.budget = c->wait_cycles ? (long long)std::min<uint64_t>(c->wait_cycles, (uint64_t)tc::DRAIN_CYCLES)
                            : tc::DRAIN_CYCLES;
  if (split > 1) {
    a.acc = ar.get<unsigned long long>(rows * cols);
    a.count = ar.get<unsigned>(tiles);
    LGS_CUDA(cudaMemsetAsync(a.acc, 0, rows * cols * 8, st));
    LGS_CUDA(cudaMemsetAsync(a.count, 0, tiles * 4, st));
  }
  // the X limb tiles and x' sums of every (row tile, chunk); 16-byte aligned arena blocks
  const size_t xt_bytes = (size_t)WT_LX * nr * WT_KC;
  uint8_t* xl = ar.get<uint8_t>(ntr * chunks * xt_bytes);
  uint32_t* xsum = ar.get<uint32_t>(ntr * chunks * nr);
  a.xl = xl;
  a.xsum = xsum;
  a.chunks = chunks;
  StageTimer t(c->prof, st, "linear_witness_tc");
  x_limbs_kernel<<<dim3((unsigned)chunks, (unsigned)ntr), 256, 0, st>>>(a, xl, xsum);
  LGS_LAUNCH_CHECK();
  const dim3 grid((unsigned)mt, (unsigned)ntr, (unsigned)split);
  k<<<grid, WT_THREADS, smem, st>>>(a);
  LGS_LAUNCH_CHECK();
}

}  // namespace lgs
