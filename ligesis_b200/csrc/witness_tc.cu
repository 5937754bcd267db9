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
// in limb 0.  sum_k x' is summed per chunk by the X pre-pass.  A value outside those ranges sets
// a flag and the caller runs the CUDA-core kernel instead (witness.cu), which handles any i64.
//
// The work is a list of units: a 128-column x NR-row output tile (D^T = W_tile X^T: M = 128
// output columns, N = NR <= 64 rows) over a K range, in chunks of 128 values of K.  Whole waves
// of tiles run unsplit; the tiles left over are split over K to fill one more wave, each split
// adding its exact int64 sum into a zeroed buffer and the last to arrive (a counter per tile)
// finishing the tile.  x_limbs_kernel converts X once per launch into the limb tiles of every
// (row tile, chunk) and zeroes the split buffers.  Two kernels take the units:
//   linear_witness_tp_kernel (rows of W an even number of values, 16-byte aligned: every GPT-2
//     layer): persistent, one CTA per SM, warp-specialised: W arrives by TMA into a ring of raw
//     boxes, eight warps convert it to limbs, one thread issues the MMAs into two alternating
//     accumulator sets in TMEM, and eight warps finish each unit while the next one streams
//   linear_witness_tc_kernel (the other layouts): one CTA per unit, its eight warps loading W
//     through registers into limbs, warp 0 issuing the MMAs, warps 0-3 finishing the unit.
// Every wait is bounded.
#include <cuda.h>

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
  // The work units: tiles [0, ta) in nsp[0] K ranges of kch[0] values each (ua units, tile
  // v % ta, range v / ta), the remaining tiles in nsp[1] ranges of kch[1] (ub units, tile
  // ta + v % (tiles - ta), range v / (tiles - ta)); v counts the units of a segment, the first
  // segment's units first, or (tail_first) the second's.  Tiles are numbered row tile x mt +
  // column tile.  The tiles from split0 on are split (nsp > 1 in their segment):
  // their K ranges add exact int64 sums into acc (nrv x 128 per tile, zeroed) and the last to
  // arrive (count per tile, zeroed) finishes the tile.
  size_t mt, tiles, ta, ua, ub, split0, units;
  int tail_first;
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

// A work unit: output tile (rt, column tile) over the K range [kb, ke) of nch chunks.
struct WtUnit {
  size_t tile, rt, c0, r0, kb, ke;
  unsigned nsplit, nch;
};
__device__ __forceinline__ WtUnit wt_unit(const WtArgs& a, size_t u) {
  WtUnit w;
  const int seg = a.tail_first ? u < a.ub : u >= a.ua;
  const size_t v = seg ? (a.tail_first ? u : u - a.ua) : (a.tail_first ? u - a.ub : u);
  const size_t nseg = seg ? a.tiles - a.ta : a.ta;
  w.tile = (seg ? a.ta : 0) + v % nseg;
  const size_t part = v / nseg;
  w.nsplit = a.nsp[seg];
  w.rt = w.tile / a.mt;
  w.c0 = (w.tile % a.mt) * WT_M;
  w.r0 = w.rt * a.nrv;
  w.kb = part * a.kch[seg];
  w.ke = min(a.inner, w.kb + a.kch[seg]);
  w.nch = (unsigned)((w.ke - w.kb + WT_KC - 1) / WT_KC);
  return w;
}

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

// Barrier 1 among the epilogue's n threads.
__device__ __forceinline__ void epi_bar(unsigned n) {
  asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory");
}

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
//     2 lane, 2 lane + 1, 64 + 2 lane, 64 + 2 lane + 1;
//   else (W[k][c]): column m = 32 (warp % 4) + lane, K offsets 8 s + 4 (warp / 4) + 0..3.
// EDGE (a tile reaching past the last column or a chunk past the end of K): every address is
// clamped into the matrix (no branch, so the loads issue back to back) and store_w_group zeroes
// the values outside it; otherwise the tile and chunk lie inside the matrix.
template <bool WT, bool EDGE>
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
      v[4 * i] = __ldg(p + (EDGE ? min(ka, ke - 1) : ka));
      v[4 * i + 1] = __ldg(p + (EDGE ? min(ka + 1, ke - 1) : ka + 1));
      v[4 * i + 2] = __ldg(p + (EDGE ? min(kb2, ke - 1) : kb2));
      v[4 * i + 3] = __ldg(p + (EDGE ? min(kb2 + 1, ke - 1) : kb2 + 1));
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

// The X side of every chunk, once per launch: for row tile blockIdx.y, the chunk of K values
// [128 blockIdx.x, 128 blockIdx.x + 128) and rows 8 blockIdx.z + warp, the three limb tiles exactly
// as the main kernel's shared memory holds them (rows below nrv data, row nrv all ones in limb 0,
// the rest zero), and each data row's sum of x' over the chunk.  A value outside 24 bits sets
// *range.  The CTAs past the chunks (blockIdx.x >= chunks, in row tile 0 and row group 0) zero
// the split tiles' sums and counters.
__global__ void __launch_bounds__(256) x_limbs_kernel(const WtArgs a, uint8_t* __restrict__ xl,
                                                      uint32_t* __restrict__ xsum) {
  // the persistent kernel launched after this one may start (its weight stream does not read
  // what this kernel writes; its readers wait for this grid)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nr = a.nr;
  const size_t chunks = a.chunks, chunk = blockIdx.x, tile = blockIdx.y;
  const size_t r0 = tile * a.nrv, k0 = chunk * WT_KC;
  if (chunk >= chunks) {
    if (blockIdx.y || blockIdx.z) return;
    const size_t nth = (size_t)(gridDim.x - chunks) * blockDim.x;
    const size_t me = (chunk - chunks) * blockDim.x + threadIdx.x;
    const size_t nt = a.tiles - a.split0, nacc = nt * a.nrv * WT_M;
    ulonglong2* acc2 = (ulonglong2*)a.acc;  // 16-byte aligned
    for (size_t i = me; i < nacc / 2; i += nth) acc2[i] = make_ulonglong2(0, 0);
    if (me == 0 && nacc % 2) a.acc[nacc - 1] = 0;
    for (size_t i = me; i < nt; i += nth) a.count[i] = 0;
    return;
  }
  const unsigned r = 8 * blockIdx.z + warp;
  if (r >= nr) return;
  uint8_t* base = xl + (tile * chunks + chunk) * (size_t)(WT_LX * nr * WT_KC);
  uint8_t* const tiles[WT_LX] = {base, base + nr * WT_KC, base + 2 * nr * WT_KC};
  bool bad = false;
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
template <bool WT, bool EDGE>
__device__ __forceinline__ uint64_t wt_produce(const WtArgs& a, WtCta& s) {
  const unsigned warp = s.warp, lane = s.lane, tid = s.tid, nr = s.nr, nchunks = s.nchunks;
  const size_t c0 = s.c0, kb = s.kb, ke = s.ke;
  uint64_t acc = 0;
  const size_t xt_bytes = (size_t)WT_LX * nr * WT_KC;
  const uint32_t row_off = WT ? tc::sw128_off(warp, (lane & 1) ? 62 + 2 * lane : 2 * lane) : 0;
  int64_t b0[8], b1[8], b2[8], b3[8];
  load_w_group<WT, EDGE>(a, c0, kb, ke, warp, lane, 0, b0);
  load_w_group<WT, EDGE>(a, c0, kb, ke, warp, lane, 1, b1);
  load_w_group<WT, EDGE>(a, c0, kb, ke, warp, lane, 2, b2);
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
    load_w_group<WT, EDGE>(a, c0, k0, ke, warp, lane, 3, b3);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 0, b0, acc);
    load_w_group<WT, EDGE>(a, c0, k0, ke, warp, lane, 4, b0);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 1, b1, acc);
    load_w_group<WT, EDGE>(a, c0, k0, ke, warp, lane, 5, b1);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 2, b2, acc);
    load_w_group<WT, EDGE>(a, c0, k0, ke, warp, lane, 6, b2);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 3, b3, acc);
    load_w_group<WT, EDGE>(a, c0, k0, ke, warp, lane, 7, b3);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 4, b0, acc);
    if (more) load_w_group<WT, EDGE>(a, c0, k1, ke, warp, lane, 0, b0);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 5, b1, acc);
    if (more) load_w_group<WT, EDGE>(a, c0, k1, ke, warp, lane, 1, b1);
    store_w_group<WT, EDGE>(a, wt_tiles, c0, k0, ke, warp, lane, row_off, 6, b2, acc);
    if (more) load_w_group<WT, EDGE>(a, c0, k1, ke, warp, lane, 2, b2);
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

__device__ __noinline__ bool lw_finish_ol(int64_t v, int64_t b, int64_t d, size_t o,
                                          int64_t* q_out, int64_t* rem_out, int64_t* y_out,
                                          uint64_t* yf_out) {
  return lw_finish_i64(v, b, d, o, q_out, rem_out, y_out, yf_out);
}

// The epilogue of one unit by the 128 x halves threads of 4 x halves warps (TMEM lane quarter
// q = warp % 4 holds output columns 32 q .. 32 q + 31 of the tile; half h of the warps of a
// quarter takes the row groups 4 h, 4 (h + halves), ...; leader: one of the threads) once its four
// accumulators at tmem_acc are complete: the ones row's entry of each accumulator is sum_k w' of
// the column (wpad: the part of it that K padding contributes), every data row recombines its
// four limb sums with the offset corrections and is finished (Q, REM, Y, encode_i64(Y)) or, for a
// split tile, added into the tile's sums, the last split to arrive finishing the tile.  Barrier 1
// synchronises the epilogue's threads.  false: a result leaves the i64 range.
__device__ __forceinline__ bool wt_epilogue(const WtArgs& a, const WtUnit& w, uint32_t tmem_acc,
                                            const unsigned long long* sx, unsigned q,
                                            unsigned h, unsigned halves, unsigned lane,
                                            bool leader, int* s_last, int64_t wpad) {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t lane_off = (uint32_t)(32 * q) << 16;
  const unsigned m = 32 * q + lane;
  const size_t c = w.c0 + m;
  const bool col_ok = c < a.cols;
  const int64_t bias = a.bias && col_ok ? __ldg(a.bias + c) : 0;
  // sum_k w' of this column: the ones row's entry of each accumulator.  (The epilogue runs in
  // bursts between waits, so its code is kept small: rows in groups of four, not unrolled.)
  int64_t sw = 0;
  {
    uint32_t v[WT_NG];
#pragma unroll
    for (int g = 0; g < WT_NG; ++g)
      v[g] = tc::tmem_ld1(tmem_acc + lane_off + (uint32_t)(g * a.nr) + a.nrv);
    tc::tmem_wait_ld();
#pragma unroll
    for (int g = 0; g < WT_NG; ++g) sw += (int64_t)v[g] << (8 * g);
  }
  // a split tile's sums: nrv rows of 128 columns
  unsigned long long* tacc =
      w.nsplit > 1 ? a.acc + (w.tile - a.split0) * a.nrv * WT_M : nullptr;
  const int64_t kv = (int64_t)(w.ke - w.kb);
  const int64_t base = kv * WT_OX * WT_OW - WT_OX * (sw - wpad);
  bool over = false;
#pragma unroll 1
  for (unsigned r4 = 4 * h; r4 < a.nrv; r4 += 4 * halves) {  // nr a multiple of 16: r4 + 3 < nr
    uint32_t v[WT_NG][4];
#pragma unroll
    for (int g = 0; g < WT_NG; ++g)
      tc::tmem_ld4(tmem_acc + lane_off + (uint32_t)(g * a.nr) + r4, v[g]);
    tc::tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const unsigned r = r4 + i;
      const size_t gr = w.r0 + r;
      if (r >= a.nrv || gr >= a.rows || !col_ok) continue;
      int64_t pv = 0;
#pragma unroll
      for (int g = 0; g < WT_NG; ++g) pv += (int64_t)v[g][i] << (8 * g);
      const int64_t val = pv - WT_OW * (int64_t)sx[r] + base;
      const size_t o = gr * a.cols + c;
      if (w.nsplit == 1)
        over |= !lw_finish_i64(val, bias, a.d, o, a.q, a.rem, a.y, a.yf);
      else
        atomicAdd(tacc + (size_t)r * WT_M + m, (unsigned long long)val);
    }
  }
  if (w.nsplit > 1) {
    // the last split of this tile to arrive finishes it from the summed buffer
    __threadfence();
    epi_bar(128 * halves);
    if (leader) *s_last = atomicAdd(a.count + (w.tile - a.split0), 1u) == w.nsplit - 1;
    epi_bar(128 * halves);
    if (*s_last) {
      __threadfence();
      // this thread's groups of four rows (4 h, 4 (h + halves), ...), four groups' loads in
      // flight at once; the finish out of line, so that this rarely run code stays small
#pragma unroll 1
      for (unsigned blk = 4 * h; blk < a.nrv; blk += 16 * halves) {
        int64_t val[16];
#pragma unroll
        for (int g = 0; g < 4; ++g)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const unsigned r = blk + 4 * halves * g + i;
            val[4 * g + i] = r < a.nrv ? (int64_t)__ldcg(tacc + (size_t)r * WT_M + m) : 0;
          }
#pragma unroll
        for (int g = 0; g < 4; ++g)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const unsigned r = blk + 4 * halves * g + i;
            const size_t gr = w.r0 + r;
            if (r >= a.nrv || gr >= a.rows || !col_ok) continue;
            over |= !lw_finish_ol(val[4 * g + i], bias, a.d, gr * a.cols + c, a.q, a.rem, a.y,
                                  a.yf);
          }
      }
    }
  }
  return !over;
}

// One CTA per unit, two per SM (the layouts the persistent kernel below does not take: rows of
// W with an odd number of values, or not 16-byte aligned).  WT: W is cols x inner (else inner x
// cols).
template <bool WT>
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
  const WtUnit wu = wt_unit(a, blockIdx.x);
  const size_t rt = wu.rt, c0 = wu.c0, kb = wu.kb, ke = wu.ke;
  const unsigned nchunks = wu.nch;
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
    const uint64_t acc = edge ? wt_produce<WT, true>(a, cs) : wt_produce<WT, false>(a, cs);
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
        if (!wt_epilogue(a, wu, tmem, sx, warp, 0, 1, lane, tid == 0, &s_last, 0))
          atomicOr(a.err, 1);
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

// ---- The persistent kernel (rows of W an even number of values, 16-byte aligned) --------------
// One CTA per SM walks the work units u = blockIdx.x, + gridDim.x, ... with its warps in roles:
//   warp 8      TMA: W's chunk of each unit as eight boxes of 16 KB (128 rows of W x 16 values
//               of K when W is transposed, else 128 rows of K x 16 columns; 128-byte swizzle,
//               zeros outside the matrix) into a ring of nraw boxes
//   warps 0-7   convert each box to limbs in the limb stage of its chunk (2 stages); thread 0
//               also fetches the chunk's X limb tiles with one bulk copy
//   warp 9      TMEM allocation; one thread issues each chunk's MMAs into the unit's accumulator
//               set (two sets of four accumulators, alternating by unit)
//   warps 10-17 epilogue of each unit (wt_epilogue; two warps per TMEM lane quarter) while the
//               next unit's MMAs run
// The raw ring keeps up to nraw x 16 KB of weights in flight per SM without holding registers.
// A K position past the end of the matrix reads as w = 0, so its w' is 2^15 (in range): its
// x' is 0 (the X tiles are zero there) and the epilogue takes 2^15 per such position off the
// ones row's sum.
constexpr int WP_WARPS = 18, WP_THREADS = WP_WARPS * 32;
constexpr unsigned WP_LOAD_WARP = 8, WP_MMA_WARP = 9, WP_EPI_WARP0 = 10;
constexpr unsigned WP_EPI_HALVES = 2;  // epilogue warps per TMEM lane quarter
constexpr uint32_t WP_BOX = 16 * WT_M * 8;  // one raw box, bytes
constexpr int WP_BOXES = WT_KC / 16;        // boxes per chunk
constexpr unsigned WP_RAW_MAX = 8;
// Shared memory besides the raw ring: limb stages, sx[2][64], barriers, the TMEM address, and
// the slack to align the base to 1024 bytes.
size_t wp_fixed_bytes(unsigned nr) {
  return WT_STAGES * wt_stage_bytes(nr) + 2 * WT_NR_MAX * 8 + 256 + 1024;
}
// TMEM columns: two sets of four nr-column accumulators, rounded up to a power of two.
__host__ __device__ constexpr uint32_t wp_tcols(unsigned nr) {
  return 8 * nr <= 128 ? 128 : (8 * nr <= 256 ? 256 : 512);
}

// A bounded wait on an mbarrier phase by every lane of the warp; true only if all saw it.
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, volatile int* fail,
                                          long long budget) {
  return __all_sync(0xffffffffu, tc::mbar_wait(bar, parity, fail, budget));
}

// One raw box of W (box b of its chunk) into the stage's two limb tiles, by warps 0-7.
//   WT: the box is 128 rows of W (output columns) x 16 values of K.  Lane (r8, qd) takes rows
//       8 warp + r8 and + 64, values 4 qd .. 4 qd + 3 (16-byte chunks 2 qd and 2 qd + 1 of the
//       row, swizzled by r8); the limb words go to row m, K byte 16 b + 4 qd.
//   else: the box is 128 rows of K x 16 output columns (16 b ..).  Lane (c8, q4) takes columns
//       c8 and c8 + 8, rows 4 kq .. 4 kq + 3 with kq = 4 warp + q4 (8-byte loads; a load's lanes
//       read 8 columns of 4 rows, two per swizzle pattern); the limb words go to row 16 b +
//       column, K byte 4 kq.
// Either way a limb store's 32 lanes hit 32 different banks.  acc collects the range check.
template <bool WT>
__device__ __forceinline__ void wp_convert(const uint8_t* box, uint8_t* const (&tiles)[WT_LW],
                                           int b, unsigned warp, unsigned lane, uint64_t& acc) {
  if constexpr (WT) {
    const unsigned r8 = lane >> 2, qd = lane & 3;
    const uint32_t row = (8 * warp + r8) * 128;
    const uint32_t rd0 = row + (((2 * qd) ^ r8) << 4), rd1 = row + (((2 * qd + 1) ^ r8) << 4);
    const uint32_t wr = row + (((uint32_t)b ^ r8) << 4) + 4 * qd;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const longlong2 v0 = *(const longlong2*)(box + rd0 + 8192 * h);
      const longlong2 v1 = *(const longlong2*)(box + rd1 + 8192 * h);
      const uint32_t e0 = w_word(v0.x, acc), e1 = w_word(v0.y, acc);
      const uint32_t e2 = w_word(v1.x, acc), e3 = w_word(v1.y, acc);
      store_limbs(tiles, wr + 8192 * h, pair_limbs(e0, e1), pair_limbs(e2, e3));
    }
  } else {
    const unsigned c8 = lane >> 2, kq = 4 * warp + (lane & 3);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const unsigned cl = c8 + 8 * h;
      uint32_t e[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const unsigned k = 4 * kq + j;
        e[j] = w_word(*(const int64_t*)(box + k * 128 + ((((cl >> 1) ^ k) & 7) << 4) +
                                        (cl & 1) * 8),
                      acc);
      }
      store_limbs(tiles, tc::sw128_off(16 * b + cl, 4 * kq), pair_limbs(e[0], e[1]),
                  pair_limbs(e[2], e[3]));
    }
  }
}

template <bool WT>
__global__ void __launch_bounds__(WP_THREADS, 1)
    linear_witness_tp_kernel(const __grid_constant__ CUtensorMap tmap_w, const WtArgs a,
                             unsigned nraw) {
  extern __shared__ uint8_t wt_smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)wt_smem_raw + 1023) & ~(uintptr_t)1023);
  const unsigned nr = a.nr;
  const size_t stage_bytes = wt_stage_bytes(nr);
  const size_t xt_bytes = (size_t)WT_LX * nr * WT_KC;
  uint8_t* raw = smem;
  uint8_t* stages = raw + (size_t)nraw * WP_BOX;
  unsigned long long* sxb = (unsigned long long*)(stages + WT_STAGES * stage_bytes);
  uint64_t* bars = (uint64_t*)(sxb + 2 * WT_NR_MAX);
  uint32_t* tmem_holder = (uint32_t*)(bars + 28);
  const uint32_t bar0 = tc::smem_u32(bars);
  auto raw_full = [&](unsigned i) { return bar0 + 8 * i; };
  auto raw_empty = [&](unsigned i) { return bar0 + 8 * (WP_RAW_MAX + i); };
  auto lim_full = [&](unsigned s) { return bar0 + 8 * (16 + s); };
  auto lim_empty = [&](unsigned s) { return bar0 + 8 * (18 + s); };
  auto xbar = [&](unsigned s) { return bar0 + 8 * (20 + s); };
  auto acc_full = [&](unsigned b) { return bar0 + 8 * (22 + b); };
  auto acc_empty = [&](unsigned b) { return bar0 + 8 * (24 + b); };
  const uint32_t drain = bar0 + 8 * 26;
  __shared__ volatile int s_fail;
  __shared__ int s_last;
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t tcols = wp_tcols(nr);

  if (tid == 0) {
    s_fail = 0;
    for (unsigned i = 0; i < nraw; ++i) {
      tc::mbar_init(raw_full(i), 1);
      tc::mbar_init(raw_empty(i), 8);  // one arrival per converter warp
    }
    for (unsigned s = 0; s < WT_STAGES; ++s) {
      tc::mbar_init(lim_full(s), 8);
      tc::mbar_init(lim_empty(s), 1);
      tc::mbar_init(xbar(s), 1);
      tc::mbar_init(acc_full(s), 1);
      tc::mbar_init(acc_empty(s), 4 * WP_EPI_HALVES);  // one arrival per epilogue warp
    }
    tc::mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == WP_MMA_WARP) {
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

  if (warp < 8) {
    // ---- converters (wp_convert)
    uint64_t acc = 0;
    unsigned rawi = 0, limi = 0, x_issued = 0;
    bool ok = true;
    // the X tiles come from x_limbs_kernel, which may still run (programmatic launch)
    if (tid == 0) asm volatile("griddepcontrol.wait;" ::: "memory");
    for (size_t u = blockIdx.x; ok && u < a.units; u += gridDim.x) {
      const WtUnit w = wt_unit(a, u);
      for (unsigned t = 0; t < w.nch; ++t, ++limi) {
        const unsigned s = limi % WT_STAGES;
        uint8_t* stage = stages + s * stage_bytes;
        if (limi >= WT_STAGES &&
            !warp_wait(lim_empty(s), ((limi / WT_STAGES) - 1) & 1, &s_fail, a.budget)) {
          if (lane == 0 && !s_fail) tc::flag_failure(&s_fail, a.err, 18);
          ok = false;
          break;
        }
        if (tid == 0) {
          const uint32_t bar = xbar(s);
          tc::mbar_arrive_tx(bar, (uint32_t)xt_bytes);
          x_issued = limi + 1;
          const uint8_t* src = a.xl + (w.rt * a.chunks + w.kb / WT_KC + t) * xt_bytes;
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
              "[%3];" ::"r"(tc::smem_u32(stage + WT_LW * WT_A_TILE)),
              "l"(src), "r"((uint32_t)xt_bytes), "r"(bar)
              : "memory");
        }
        uint8_t* const tiles[WT_LW] = {stage, stage + WT_A_TILE};
#pragma unroll 1
        for (int b = 0; b < WP_BOXES; ++b, ++rawi) {
          const unsigned slot = rawi % nraw;
          if (!warp_wait(raw_full(slot), (rawi / nraw) & 1, &s_fail, a.budget)) {
            if (lane == 0 && !s_fail) tc::flag_failure(&s_fail, a.err, 21);
            ok = false;
            break;
          }
          wp_convert<WT>(raw + (size_t)slot * WP_BOX, tiles, b, warp, lane, acc);
          __syncwarp();
          if (lane == 0) tc::mbar_arrive(raw_empty(slot));
        }
        if (!ok) break;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(lim_full(s));
      }
    }
    if (acc >> 16) atomicExch(a.range, 1);
    if (tid == 0) {
      // the newest X copy of each stage may still be in flight: wait for it before exiting
      for (unsigned g = x_issued > WT_STAGES ? x_issued - WT_STAGES : 0; g < x_issued; ++g)
        if (!tc::mbar_wait_drain(xbar(g % WT_STAGES), (g / WT_STAGES) & 1)) atomicExch(a.err, 20);
    }
  }
  else if (warp == WP_LOAD_WARP) {
    // ---- TMA: W transposed: box (16 values of K from kb + 128 t + 16 b) x (128 rows of W from
    // c0); else (16 columns from c0 + 16 b) x (128 rows of K from kb + 128 t)
    if (lane == 0) {
      unsigned rawi = 0;
      bool ok = true;
      for (size_t u = blockIdx.x; ok && u < a.units; u += gridDim.x) {
        const WtUnit w = wt_unit(a, u);
        for (unsigned t = 0; ok && t < w.nch; ++t)
          for (int b = 0; b < WP_BOXES; ++b, ++rawi) {
            const unsigned slot = rawi % nraw;
            if (rawi >= nraw &&
                !tc::mbar_wait(raw_empty(slot), ((rawi / nraw) - 1) & 1, &s_fail, a.budget)) {
              if (!s_fail) tc::flag_failure(&s_fail, a.err, 22);
              ok = false;
              break;
            }
            const uint32_t bar = raw_full(slot);
            tc::mbar_arrive_tx(bar, WP_BOX);
            const int x = WT ? (int)(w.kb + (size_t)t * WT_KC + 16 * b) : (int)(w.c0 + 16 * b);
            const int y = WT ? (int)w.c0 : (int)(w.kb + (size_t)t * WT_KC);
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                "[%0], [%1, {%2, %3}], [%4];" ::"r"(tc::smem_u32(raw + (size_t)slot * WP_BOX)),
                "l"((uint64_t)&tmap_w), "r"(x), "r"(y), "r"(bar)
                : "memory");
          }
      }
      // the newest load of each slot may still be in flight: wait for it before exiting
      for (unsigned g = rawi > nraw ? rawi - nraw : 0; g < rawi; ++g)
        if (!tc::mbar_wait_drain(raw_full(g % nraw), (g / nraw) & 1)) atomicExch(a.err, 24);
    }
  } else if (warp == WP_MMA_WARP) {
    // ---- MMA issue: unit i accumulates in set i % 2 once the epilogue has drained that set;
    // each chunk is 4 K steps x 6 limb pairs, pair (i, j) into accumulator i + j
    if (lane == 0) {
      unsigned limi = 0, i = 0;
      bool ok = true;
      const uint32_t idesc = tc::idesc_u8(WT_M, nr);
      for (size_t u = blockIdx.x; ok && u < a.units; u += gridDim.x, ++i) {
        const WtUnit w = wt_unit(a, u);
        const unsigned b = i & 1;
        if (i >= 2 && !tc::mbar_wait(acc_empty(b), ((i / 2) - 1) & 1, &s_fail, a.budget)) {
          if (!s_fail) tc::flag_failure(&s_fail, a.err, 23);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t dacc = tmem + b * WT_NG * nr;
        for (unsigned t = 0; t < w.nch; ++t, ++limi) {
          const unsigned s = limi % WT_STAGES, ph = (limi / WT_STAGES) & 1;
          if (!tc::mbar_wait(lim_full(s), ph, &s_fail, a.budget) ||
              !tc::mbar_wait(xbar(s), ph, &s_fail, a.budget)) {
            if (!s_fail) tc::flag_failure(&s_fail, a.err, 16);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sa = tc::smem_u32(stages + s * stage_bytes);
          const uint32_t sb = sa + (uint32_t)(WT_LW * WT_A_TILE);
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
#pragma unroll
            for (int li = 0; li < WT_LX; ++li)
#pragma unroll
              for (int lj = 0; lj < WT_LW; ++lj) {
                // the first pair of each accumulator in the unit's first K step overwrites it
                const bool first = t == 0 && ks == 0 && (lj == 1 || li == 0);
                tc::mma_i8(dacc + (uint32_t)((li + lj) * nr),
                           tc::sw128_desc(sa + (uint32_t)(lj * WT_A_TILE) + 32 * ks),
                           tc::sw128_desc(sb + (uint32_t)(li * nr * WT_KC) + 32 * ks), idesc,
                           first ? 0u : 1u);
              }
          tc::mma_commit(lim_empty(s));
        }
        if (ok) tc::mma_commit(acc_full(b));
      }
      // every MMA issued so far has completed once this arrives: wait before the TMEM is freed
      tc::mma_commit(drain);
      if (!tc::mbar_wait_drain(drain, 0)) atomicExch(a.err, 17);
    }
  } else {
    // ---- epilogue (warps 10-17: TMEM lane quarter warp % 4, row groups of half (warp - 10) / 4)
    const unsigned q = warp & 3, h = (warp - WP_EPI_WARP0) / 4, et = tid - 32 * WP_EPI_WARP0;
    // x' sums, zeroed split sums and counters: written by x_limbs_kernel
    asm volatile("griddepcontrol.wait;" ::: "memory");
    unsigned i = 0;
    for (size_t u = blockIdx.x; u < a.units; u += gridDim.x, ++i) {
      const WtUnit w = wt_unit(a, u);
      const unsigned b = i & 1;
      unsigned long long* sx = sxb + b * WT_NR_MAX;
      if (et < nr) {  // this unit's sums of x' per row, from the per-chunk sums
        unsigned long long sum = 0;
        for (unsigned t = 0; t < w.nch; ++t)
          sum += a.xsum[(w.rt * a.chunks + w.kb / WT_KC + t) * nr + et];
        sx[et] = sum;
      }
      const bool got = tc::mbar_wait(acc_full(b), (i / 2) & 1, &s_fail, a.budget);
      uint32_t all;
      asm volatile(
          "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, 1, %2, p;\n"
          " selp.u32 %0, 1, 0, q;\n}\n"
          : "=r"(all)
          : "r"((uint32_t)got), "r"(128 * WP_EPI_HALVES)
          : "memory");
      if (!all) {
        if (!s_fail) tc::flag_failure(&s_fail, a.err, 19);
        break;
      }
      const int64_t wpad = (int64_t)((size_t)w.nch * WT_KC - (w.ke - w.kb)) << 15;
      if (!wt_epilogue(a, w, tmem + b * WT_NG * nr, sx, q, h, WP_EPI_HALVES, lane, et == 0, &s_last,
                       wpad))
        atomicOr(a.err, 1);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(acc_empty(b));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == WP_MMA_WARP) {
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
  auto kp = w_transposed ? linear_witness_tp_kernel<true> : linear_witness_tp_kernel<false>;
  int nsm = 148, smem_sm = 0, smem_optin = 0;
  LGS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
  LGS_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                                  c->device));
  LGS_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                  c->device));
  // as many 16 KB boxes of weights in flight as shared memory holds beside the limb stages
  const size_t fixed = wp_fixed_bytes(nr);
  const unsigned nraw =
      (size_t)smem_optin > fixed + 1024
          ? (unsigned)std::min<size_t>(WP_RAW_MAX, ((size_t)smem_optin - fixed - 1024) / WP_BOX)
          : 0;
  // W's rows an even number of values and 16-byte aligned, and room for a ring of at least two
  // boxes: the persistent kernel (its weights arrive by TMA); otherwise one CTA per unit, two
  // per SM
  const bool persistent = (w_transposed ? inner % 2 == 0 : cols % 2 == 0) &&
                          (((uintptr_t)dw & 15) == 0) && nraw >= 2;
  size_t smem, slots, fixed_cost;
  CUtensorMap tm{};  // encoded before the first launch, so the launches follow back to back
  auto k = w_transposed ? linear_witness_tc_kernel<true> : linear_witness_tc_kernel<false>;
  if (persistent) {
    smem = fixed + (size_t)nraw * WP_BOX;
    LGS_CUDA(cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // boxes of 128 rows x 16 values: rows of W (transposed) or rows of K
    if (w_transposed)
      make_i64_tmap(dw, cols, inner, WT_M, &tm);
    else
      make_i64_tmap(dw, inner, cols, WT_KC, &tm);
    slots = c->witness_ctas ? c->witness_ctas : (size_t)nsm;
    fixed_cost = 1;  // a unit's start and epilogue overlap the neighbouring units' streams
  } else {
    smem = wt_smem_bytes(nr);
    LGS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // two CTAs per SM need the largest shared-memory carveout
    LGS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared));
    // resident CTAs per SM: the launch bounds cap registers for two; shared memory decides
    const size_t per_sm = 2 * (smem + 1024) <= (size_t)smem_sm ? 2 : 1;
    slots = c->witness_ctas ? c->witness_ctas : per_sm * nsm;
    fixed_cost = 3;  // start-up, and the epilogue with a split's atomics and finish
  }
  const size_t mt = (cols + WT_M - 1) / WT_M, tiles = mt * ntr;
  const size_t chunks = (inner + WT_KC - 1) / WT_KC;
  // K splits: the fewest that minimise (waves of units) x (chunks per unit + the fixed cost of
  // a unit), and enough that no unit sums more than WT_KMAX values of K.  Either one split for
  // every tile, or (more tiles than resident CTAs) whole waves of tiles with the fewest splits
  // and the remaining tiles split apart to fill one last wave.
  const size_t min_split = (inner + WT_KMAX - 1) / WT_KMAX;
  auto best_split = [&](size_t n, size_t& cost) {
    size_t split = min_split;
    cost = SIZE_MAX;
    for (size_t sp = min_split; sp <= std::min<size_t>(chunks, 64); ++sp) {
      const size_t cst = ((n * sp + slots - 1) / slots) * ((chunks + sp - 1) / sp + fixed_cost);
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
  a.budget = c->wait_cycles
                 ? (long long)std::min<uint64_t>(c->wait_cycles, (uint64_t)tc::DRAIN_CYCLES)
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
  a.ub = (tiles - ta) * a.nsp[1];
  // one CTA per unit: the long units first (the short ones fill the last wave); persistent:
  // each CTA's split units first, so that its last epilogue is a whole tile's (no atomics)
  a.tail_first = persistent ? 1 : 0;
  const size_t units = a.ua + a.ub;
  a.units = units;
  StageTimer t(c->prof, st, "linear_witness_tc");
  if (a.split0 < tiles) {  // zeroed by x_limbs_kernel
    const size_t nsplit_tiles = tiles - a.split0;
    a.acc = ar.get<unsigned long long>(nsplit_tiles * nrv * WT_M);
    a.count = ar.get<unsigned>(nsplit_tiles);
  }
  // the X limb tiles and x' sums of every (row tile, chunk); 16-byte aligned arena blocks
  const size_t xt_bytes = (size_t)WT_LX * nr * WT_KC;
  uint8_t* xl = ar.get<uint8_t>(ntr * chunks * xt_bytes);
  uint32_t* xsum = ar.get<uint32_t>(ntr * chunks * nr);
  a.xl = xl;
  a.xsum = xsum;
  a.chunks = chunks;
  // CTAs for the zeroing: four 16-byte stores per thread
  const size_t nacc = a.split0 < tiles ? (tiles - a.split0) * nrv * WT_M : 0;
  const size_t zctas = nacc ? std::min<size_t>(4 * (size_t)nsm, (nacc + 2047) / 2048) : 0;
  x_limbs_kernel<<<dim3((unsigned)(chunks + zctas), (unsigned)ntr, (nr + 7) / 8), 256, 0, st>>>(
      a, xl, xsum);
  LGS_LAUNCH_CHECK();
  if (persistent) {
    // launched while x_limbs_kernel runs: its weight stream starts at once, the threads that
    // read the X side wait for that grid (griddepcontrol.wait)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)std::min(units, slots));
    cfg.blockDim = dim3(WP_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    LGS_CUDA(cudaLaunchKernelEx(&cfg, kp, tm, a, nraw));
  } else {
    k<<<(unsigned)units, WT_THREADS, smem, st>>>(a);
  }
  LGS_LAUNCH_CHECK();
}

}  // namespace lgs
