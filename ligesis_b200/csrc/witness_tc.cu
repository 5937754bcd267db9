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
  size_t rows, inner, cols;
  unsigned nr, nrv;  // MMA N, and the x rows of a row tile (nrv < nr: one ones row)
  int wt;
  int64_t d;
  int64_t *q, *rem, *y;
  uint64_t* yf;
  // The work units (one CTA each): tiles [0, ta) in nsp[0] K ranges of kch[0] values each
  // (units [0, ua), tile u % ta, range u / ta), the remaining tiles in nsp[1] ranges of kch[1]
  // (tile ta + v % (tiles - ta), range v / (tiles - ta), v = u - ua).  Tiles are numbered row
  // tile x mt + column tile.  The tiles from split0 on are split (nsp > 1 in their segment):
  // their K ranges add exact int64 sums into acc (nrv x 128 per tile, zeroed) and the last to
  // arrive (count per tile, zeroed) finishes the tile.
  size_t mt, tiles, ta, ua, split0;
  size_t kch[2];
  unsigned nsp[2];
  unsigned long long* acc;
  unsigned* count;
  int* err;                 // 1: a result leaves the i64 range; >= 16: a bounded wait gave up
  int* range;               // an operand outside the limb encodings
  long long budget;
  const uint8_t* xl;        // the X limb tiles of every (row tile, chunk), x_limbs_kernel
  const uint32_t* xsum;     // sum of x' per (row tile, chunk, row)
  size_t chunks;            // chunks of 128 values of K in the whole inner dimension
};

// x' = x + 2^23 of a value in range, 0 for padding (outside the matrix); flags a value that
// does not fit 24 bits.
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

// w' = w + 2^15 as a 32-bit word: its low 16 bits are the two limbs of a weight in range.  acc
// collects the OR of every w' as 64 bits, so acc >> 16 != 0 at the end flags a weight outside
// [-2^15, 2^15).  Padding (valid false) encodes as 0.
__device__ __forceinline__ uint32_t w_word(int64_t v, uint64_t& acc) {
  const uint64_t e = (uint64_t)v + (uint64_t)WT_OW;
  acc |= e;
  return (uint32_t)e;
}
__device__ __forceinline__ uint32_t w_word(int64_t v, bool valid, uint64_t& acc) {
  const uint64_t e = valid ? (uint64_t)v + (uint64_t)WT_OW : 0;
  acc |= e;
  return (uint32_t)e;
}
// The limb 0 and limb 1 words of four consecutive K values from their w' words: two byte
// permutes interleave the pairs (e0.b0 e1.b0 e0.b1 e1.b1), two more split the limbs.
__device__ __forceinline__ uint32_t pair_limbs(uint32_t e0, uint32_t e1) {
  return __byte_perm(e0, e1, 0x5140);
}
__device__ __forceinline__ void store_limbs(uint8_t* const (&tiles)[WT_LW], uint32_t off,
                                            uint32_t lo_pair, uint32_t hi_pair) {
  *(uint32_t*)(tiles[0] + off) = __byte_perm(lo_pair, hi_pair, 0x5410);
  *(uint32_t*)(tiles[1] + off) = __byte_perm(lo_pair, hi_pair, 0x7632);
}

// Group q (steps 2q, 2q + 1 of 16) of the W values this thread stages for the chunk at k0:
//   w transposed (W[c][k]): step s is output column m = 8 s + warp, the values at K offsets
//     2 lane, 2 lane + 1, 64 + 2 lane, 64 + 2 lane + 1 (two 16-byte loads when vec);
//   else (W[k][c]): column m = 32 (warp % 4) + lane, K offsets 8 s + 4 (warp / 4) + 0..3.
// EDGE (a tile reaching past the last column or a chunk past the end of K): every address is
// clamped into the matrix (no branch, so the loads issue back to back) and store_w_group zeroes
// the values outside it; otherwise the tile and chunk lie inside the matrix.
template <bool WT, bool VEC, bool EDGE>
__device__ __forceinline__ void load_w_group(const WtArgs& a, size_t c0, size_t k0, size_t ke,
                                             unsigned warp, unsigned lane, int q,
                                             int64_t (&v)[8]) {
  if constexpr (WT) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const size_t c0i = c0 + 8 * (2 * q + i) + warp;
      const size_t c = EDGE ? min(c0i, a.cols - 1) : c0i;
      const int64_t* p = a.w + c * a.inner;
      const size_t ka = k0 + 2 * lane, kb2 = k0 + 64 + 2 * lane;
      if constexpr (VEC) {  // inner even: ke - 2 >= k0 is even: both 16-byte loads stay in the row
        const longlong2 x = __ldg((const longlong2*)(p + (EDGE ? min(ka, ke - 2) : ka)));
        const longlong2 y = __ldg((const longlong2*)(p + (EDGE ? min(kb2, ke - 2) : kb2)));
        v[4 * i] = x.x, v[4 * i + 1] = x.y, v[4 * i + 2] = y.x, v[4 * i + 3] = y.y;
      } else {
        v[4 * i] = __ldg(p + (EDGE ? min(ka, ke - 1) : ka));
        v[4 * i + 1] = __ldg(p + (EDGE ? min(ka + 1, ke - 1) : ka + 1));
        v[4 * i + 2] = __ldg(p + (EDGE ? min(kb2, ke - 1) : kb2));
        v[4 * i + 3] = __ldg(p + (EDGE ? min(kb2 + 1, ke - 1) : kb2 + 1));
      }
    }
  } else {
    const size_t ci = c0 + 32 * (warp & 3) + lane;
    const size_t c = EDGE ? min(ci, a.cols - 1) : ci;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const size_t kk = k0 + 8 * (2 * q + i) + 4 * (warp >> 2);
#pragma unroll
      for (int j = 0; j < 4; ++j)
        v[4 * i + j] = __ldg(a.w + (EDGE ? min(kk + j, ke - 1) : kk + j) * a.cols + c);
    }
  }
}
// The same group as limbs in the stage's two W tiles.  row_off: this thread's byte offset in
// the tile of its first row (w transposed: sw128_off(warp, K byte of the lane's four values);
// the rows 8 j further are 1024 j further, the swizzle depending on the row mod 8 only).
template <bool WT, bool EDGE>
__device__ __forceinline__ void store_w_group(const WtArgs& a, uint8_t* const (&tiles)[WT_LW],
                                              size_t c0, size_t k0, size_t ke, unsigned warp,
                                              unsigned lane, uint32_t row_off, int q,
                                              const int64_t (&v)[8], uint64_t& acc) {
  if constexpr (WT) {
    const bool odd = lane & 1;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const unsigned m = 8 * (2 * q + i) + warp;
      uint32_t e[4];
      if constexpr (EDGE) {
        const bool ok = c0 + m < a.cols;
        const size_t ka = k0 + 2 * lane, kb2 = k0 + 64 + 2 * lane;
        e[0] = w_word(v[4 * i], ok && ka < ke, acc);
        e[1] = w_word(v[4 * i + 1], ok && ka + 1 < ke, acc);
        e[2] = w_word(v[4 * i + 2], ok && kb2 < ke, acc);
        e[3] = w_word(v[4 * i + 3], ok && kb2 + 1 < ke, acc);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) e[j] = w_word(v[4 * i + j], acc);
      }
      // lane pairs swap halves: even lanes own K offsets 4j.., odd lanes 64 + 4j..
      const uint32_t lo = pair_limbs(e[0], e[1]), hi = pair_limbs(e[2], e[3]);
      const uint32_t other = __shfl_xor_sync(0xffffffffu, odd ? lo : hi, 1);
      store_limbs(tiles, row_off + 1024u * (2 * q + i), odd ? other : lo, odd ? hi : other);
    }
  } else {
    const unsigned m = 32 * (warp & 3) + lane;
    const bool ok = !EDGE || c0 + m < a.cols;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const unsigned kk = 8 * (2 * q + i) + 4 * (warp >> 2);
      uint32_t e[4];
#pragma unroll
      for (int j = 0; j < 4; ++j)
        e[j] = EDGE ? w_word(v[4 * i + j], ok && k0 + kk + j < ke, acc) : w_word(v[4 * i + j], acc);
      store_limbs(tiles, tc::sw128_off(m, kk), pair_limbs(e[0], e[1]), pair_limbs(e[2], e[3]));
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

// What the producer loop shares with the rest of its CTA.
struct WtCta {
  uint8_t* smem;
  size_t stage_bytes;
  uint32_t full0, empty0, xbar0, accf;
  volatile int* fail;
  uint32_t tmem;
  size_t c0, kb, ke;
  unsigned nchunks, nr, rt, tid, warp, lane;
  unsigned x_issued;  // thread 0: X tile copies issued
};

// The producers' loop over the chunks of a CTA's K range (warps 0-7): the W tile (128 output
// columns) of each chunk as limbs, in eight groups of eight values per thread; the loads run
// three groups ahead of the stores (a ring of four register buffers, across chunk boundaries).
// Thread 0 also fetches the chunk's X limb tiles (made once per launch by x_limbs_kernel) with
// one bulk copy, and once every producer has staged a chunk, thread 0 issues its MMAs.  Returns
// the OR of this thread's w' words (the range check).
template <bool WT, bool VEC, bool EDGE>
__device__ __forceinline__ uint64_t wt_produce(const WtArgs& a, WtCta& s) {
  const unsigned warp = s.warp, lane = s.lane, tid = s.tid, nr = s.nr, nchunks = s.nchunks;
  const size_t c0 = s.c0, kb = s.kb, ke = s.ke;
  uint64_t acc = 0;
  const size_t xt_bytes = (size_t)WT_LX * nr * WT_KC;
  const uint32_t row_off = WT ? tc::sw128_off(warp, (lane & 1) ? 62 + 2 * lane : 2 * lane) : 0;
  int64_t b0[8], b1[8], b2[8], b3[8];
  load_w_group<WT, VEC, EDGE>(a, c0, kb, ke, warp, lane, 0, b0);
  load_w_group<WT, VEC, EDGE>(a, c0, kb, ke, warp, lane, 1, b1);
  load_w_group<WT, VEC, EDGE>(a, c0, kb, ke, warp, lane, 2, b2);
  for (unsigned t = 0; t < nchunks; ++t) {
    const unsigned st = t % WT_STAGES;
    const size_t k0 = kb + (size_t)t * WT_KC, k1 = k0 + WT_KC;
    const bool more = t + 1 < nchunks;
    if (t >= WT_STAGES) {  // one lane waits, so the warp decides as one (it shuffles below)
      bool ok = true;
      if (lane == 0)
        ok = tc::mbar_wait(s.empty0 + 8 * st, ((t / WT_STAGES) - 1) & 1, s.fail, a.budget);
      if (!__shfl_sync(0xffffffffu, ok, 0)) {
        if (lane == 0 && !*s.fail) tc::flag_failure(s.fail, a.err, 18);
        break;
      }
    }
    uint8_t* stage = s.smem + st * s.stage_bytes;
    uint8_t* const wt_tiles[WT_LW] = {stage, stage + WT_A_TILE};
    if (tid == 0) {
      const uint32_t bar = s.xbar0 + 8 * st;
      tc::mbar_arrive_tx(bar, (uint32_t)xt_bytes);
      s.x_issued = t + 1;
      const uint8_t* src = a.xl + (s.rt * a.chunks + kb / WT_KC + t) * xt_bytes;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
          "[%3];" ::"r"(tc::smem_u32(stage + WT_LW * WT_A_TILE)),
          "l"(src), "r"((uint32_t)xt_bytes), "r"(bar)
          : "memory");
    }
    load_w_group<WT, VEC, EDGE>(a, c0, k0, ke, warp, lane, 3, b3);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 0, b0, acc);
    load_w_group<WT, VEC, EDGE>(a, c0, k0, ke, warp, lane, 4, b0);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 1, b1, acc);
    load_w_group<WT, VEC, EDGE>(a, c0, k0, ke, warp, lane, 5, b1);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 2, b2, acc);
    load_w_group<WT, VEC, EDGE>(a, c0, k0, ke, warp, lane, 6, b2);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 3, b3, acc);
    load_w_group<WT, VEC, EDGE>(a, c0, k0, ke, warp, lane, 7, b3);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 4, b0, acc);
    if (more) load_w_group<WT, VEC, EDGE>(a, c0, k1, ke, warp, lane, 0, b0);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 5, b1, acc);
    if (more) load_w_group<WT, VEC, EDGE>(a, c0, k1, ke, warp, lane, 1, b1);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 6, b2, acc);
    if (more) load_w_group<WT, VEC, EDGE>(a, c0, k1, ke, warp, lane, 2, b2);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 7, b3, acc);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc::mbar_arrive(s.full0 + 8 * st);
    if (warp == 0) {
      // MMA issue: once every producer has staged the chunk, 4 K steps x 6 limb pairs, pair
      // (i, j) into accumulator i + j; the commit frees the stage
      bool ok = true;
      if (lane == 0)
        ok = tc::mbar_wait(s.full0 + 8 * st, (t / WT_STAGES) & 1, s.fail, a.budget) &&
             tc::mbar_wait(s.xbar0 + 8 * st, (t / WT_STAGES) & 1, s.fail, a.budget);
      if (!__shfl_sync(0xffffffffu, ok, 0)) {
        if (lane == 0 && !*s.fail) tc::flag_failure(s.fail, a.err, 16);
        break;
      }
      if (lane == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t idesc = tc::idesc_u8(WT_M, nr);
        const uint32_t sa = tc::smem_u32(stage);
        const uint32_t sb = sa + (uint32_t)(WT_LW * WT_A_TILE);
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
#pragma unroll
          for (int i = 0; i < WT_LX; ++i)
#pragma unroll
            for (int j = 0; j < WT_LW; ++j) {
              // the first pair of each accumulator in the first K step overwrites it
              const bool first = t == 0 && ks == 0 && (j == 1 || i == 0);
              tc::mma_i8(s.tmem + (uint32_t)((i + j) * nr),
                         tc::sw128_desc(sa + (uint32_t)(j * WT_A_TILE) + 32 * ks),
                         tc::sw128_desc(sb + (uint32_t)(i * nr * WT_KC) + 32 * ks), idesc,
                         first ? 0u : 1u);
            }
        tc::mma_commit(s.empty0 + 8 * st);
        if (t + 1 == nchunks) tc::mma_commit(s.accf);
      }
      __syncwarp();
    }
  }
  return acc;
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
  // this CTA's work unit
  const size_t u = blockIdx.x;
  const int seg = u >= a.ua;
  const size_t nseg = seg ? a.tiles - a.ta : a.ta, v = seg ? u - a.ua : u;
  const size_t tile = (seg ? a.ta : 0) + v % nseg, part = v / nseg;
  const unsigned nsplit = a.nsp[seg];
  const size_t rt = tile / a.mt, c0 = (tile % a.mt) * WT_M, r0 = rt * a.nrv;
  const size_t kb = part * a.kch[seg], ke = min(a.inner, kb + a.kch[seg]);
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
    // ---- producers (the whole tile inside the matrix, or not)
    WtCta cs{smem, stage_bytes, full0, empty0, xbar0, accf, &s_fail, tmem, c0, kb, ke, nchunks,
             nr, (unsigned)rt, tid, warp, lane, 0};
    const bool edge = c0 + WT_M > a.cols || (ke - kb) % WT_KC != 0;
    const uint64_t acc = edge ? wt_produce<WT, VEC, true>(a, cs) : wt_produce<WT, VEC, false>(a, cs);
    x_issued = cs.x_issued;
    if (acc >> 16) atomicExch(a.range, 1);
    // this CTA's sums of x' per row, from the per-chunk sums
    if (tid < nr) {
      unsigned long long sum = 0;
      for (unsigned t = 0; t < nchunks; ++t)
        sum += a.xsum[(rt * a.chunks + kb / WT_KC + t) * nr + tid];
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
        // a split tile's sums: nrv rows of 128 columns
        unsigned long long* tacc =
            nsplit > 1 ? a.acc + (tile - a.split0) * a.nrv * WT_M : nullptr;
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
            if (nsplit == 1)
              over |= !lw_finish(Acc128{(uint64_t)val, (uint64_t)(val >> 63)}, a.bias, c, a.d, o,
                                 a.q, a.rem, a.y, a.yf);
            else
              atomicAdd(tacc + (size_t)r * WT_M + m, (unsigned long long)val);
          }
        }
        if (nsplit > 1) {
          // the last split of this tile to arrive finishes it from the summed buffer
          __threadfence();
          epi_bar();
          if (tid == 0) s_last = atomicAdd(a.count + (tile - a.split0), 1u) == nsplit - 1;
          epi_bar();
          if (s_last) {
            __threadfence();
            for (unsigned r = 0; r < a.nrv; ++r) {
              const size_t gr = r0 + r;
              if (gr >= a.rows || !col_ok) continue;
              const size_t o = gr * a.cols + c;
              const int64_t val = (int64_t)__ldcg(tacc + (size_t)r * WT_M + m);
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
  const size_t slots = c->witness_ctas ? c->witness_ctas : per_sm * nsm;
  const size_t mt = (cols + WT_M - 1) / WT_M, tiles = mt * ntr;
  const size_t chunks = (inner + WT_KC - 1) / WT_KC;
  // K splits: the fewest that minimise (waves of CTAs) x (chunks per CTA + the fixed cost of a
  // CTA, about three chunks with the split epilogue's atomics and finish), and enough that no
  // CTA sums more than WT_KMAX values of K.  Either one split for every tile, or (more tiles
  // than resident CTAs) whole waves of tiles with the fewest splits and the remaining tiles
  // split apart to fill one last wave.
  const size_t min_split = (inner + WT_KMAX - 1) / WT_KMAX;
  auto best_split = [&](size_t n, size_t& cost) {
    size_t split = min_split;
    cost = SIZE_MAX;
    for (size_t sp = min_split; sp <= std::min<size_t>(chunks, 64); ++sp) {
      const size_t cst = ((n * sp + slots - 1) / slots) * ((chunks + sp - 1) / sp + 3);
      if (cst < cost) cost = cst, split = sp;
    }
    return split;
  };
  size_t cost_all, cost_a = 0, cost_b = 0;
  size_t sp_a = best_split(tiles, cost_all), sp_b = 1, ta = tiles;
  if (tiles > slots && tiles % slots) {
    const size_t ta2 = tiles / slots * slots;
    const size_t sa = best_split(ta2, cost_a), sb = best_split(tiles - ta2, cost_b);
    if (cost_a + cost_b < cost_all) ta = ta2, sp_a = sa, sp_b = sb;
  }
  Arena& ar = c->arena;
  WtArgs a{dx, dw, db, rows, inner, cols, nr, nrv, w_transposed ? 1 : 0, divisor, dq, dr, dy, df};
  a.err = derr;
  a.range = drange;
  a.budget = c->wait_cycles ? (long long)std::min<uint64_t>(c->wait_cycles, (uint64_t)tc::DRAIN_CYCLES)
                            : tc::DRAIN_CYCLES;
  const size_t sps[2] = {sp_a, sp_b};
  for (int g = 0; g < 2; ++g) {
    a.kch[g] = (chunks + sps[g] - 1) / sps[g] * WT_KC;
    a.nsp[g] = (unsigned)((inner + a.kch[g] - 1) / a.kch[g]);
  }
  a.mt = mt;
  a.tiles = tiles;
  a.ta = ta;
  a.ua = ta * a.nsp[0];
  a.split0 = a.nsp[0] > 1 ? 0 : (ta < tiles && a.nsp[1] > 1 ? ta : tiles);
  const size_t units = a.ua + (tiles - ta) * a.nsp[1];
  StageTimer t(c->prof, st, "linear_witness_tc");
  if (a.split0 < tiles) {
    const size_t nsplit_tiles = tiles - a.split0;
    a.acc = ar.get<unsigned long long>(nsplit_tiles * nrv * WT_M);
    a.count = ar.get<unsigned>(nsplit_tiles);
    LGS_CUDA(cudaMemsetAsync(a.acc, 0, nsplit_tiles * nrv * WT_M * 8, st));
    LGS_CUDA(cudaMemsetAsync(a.count, 0, nsplit_tiles * 4, st));
  }
  // the X limb tiles and x' sums of every (row tile, chunk); 16-byte aligned arena blocks
  const size_t xt_bytes = (size_t)WT_LX * nr * WT_KC;
  uint8_t* xl = ar.get<uint8_t>(ntr * chunks * xt_bytes);
  uint32_t* xsum = ar.get<uint32_t>(ntr * chunks * nr);
  a.xl = xl;
  a.xsum = xsum;
  a.chunks = chunks;
  x_limbs_kernel<<<dim3((unsigned)chunks, (unsigned)ntr), 256, 0, st>>>(a, xl, xsum);
  LGS_LAUNCH_CHECK();
  k<<<(unsigned)units, WT_THREADS, smem, st>>>(a);
  LGS_LAUNCH_CHECK();
}

}  // namespace lgs
