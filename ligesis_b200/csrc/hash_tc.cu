// Subset-sum hash H = A * B (pcs/src/subset_sum.rs:43-67, called at pcs/src/ligesis.rs:302) on
// the 5th-generation tensor cores, fused with the Merkle leaf hashes of H's columns
// (pcs/src/ligesis.rs:306-313).
//
// Exactness: A's canonical 64-bit entries are split into byte limbs, Alimb[8r + l][k] = byte l of
// A[r][k], and B[64 i + b][j] = bit b of the RS codeword word F'[i][j].  S_l = Alimb_l * B is an
// exact int32 sum (terms <= 255, at most 64 * 2^13 of them), and H[r][j] = sum_l 2^(8l) S_l mod p
// is recombined exactly in 128-bit arithmetic.  K is stored permuted inside each aligned group of
// 32 (the same permutation in A's limb columns and B's rows, so the products are unchanged): it
// lets the producers spread a word's bits into bytes with a shift and a mask per 4 bytes.
//
// Persistent CTAs (one per SM) walk the 256-column tiles.  A tile is all 256 limb rows (two
// M = 128 accumulators in TMEM, 2 x 256 columns = the SM's 512 TMEM columns) by 256 codeword
// columns (N = 256); K advances 128 bytes (two codeword rows) per pipeline stage, 3 stages.
//   warp 0      TMA producer: the 256 x 128-byte A-limb tile, SWIZZLE_128B, no multicast
//   warp 1      TMEM allocation, and one thread issuing tcgen05.mma.kind::i8 (M128 N256 K32)
//   warps 2-5   B producers: expand 2 x 256 codeword words (loaded three stages ahead) into the
//               256 x 128-byte K-major SWIZZLE_128B bit tile
//   warps 6-13  epilogue, two sets of four warps taking alternate 8-column steps: tcgen05.ld
//               the int32 limb sums, recombine mod p, write H, release the
//               accumulators; then hash each 256-byte column leaf with BLAKE3 (reading H back
//               from L2) while the MMAs of the next tile run.
// Every mbarrier wait is bounded by a clock budget and watches a CTA-wide failure flag; on a
// timeout the CTA records an error code, every role stops issuing work, the MMA thread waits
// (bounded) for the MMAs it issued, the TMA thread waits (bounded) for the A-limb copies it
// issued (each stage's copy completes on its own barrier, so this wait does not depend on the
// other roles), and the TMEM is freed before the CTA exits.  The budget of the role waits is a
// kernel argument (lgs_set_wait_budget shortens it to test this path); the two drain waits
// always keep the long default.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "blake3.cuh"
#include "kernels.cuh"
#include "tcgen05.cuh"

namespace lgs {

namespace {
constexpr int TC_N = 256;
constexpr int H_ROWS = 32;  // digest rows (C)
constexpr int TC_KB = 128;
constexpr int TC_STAGES = 3;
constexpr int A_TILE = 256 * TC_KB;
constexpr int B_TILE = TC_N * TC_KB;
constexpr int STAGE_BYTES = A_TILE + B_TILE;
constexpr int NPROD = 128;
constexpr int NEPI = 256;  // epilogue threads: two sets of four warps, one per TMEM lane quarter
constexpr int NTHREADS = 64 + NPROD + NEPI;
constexpr int TMEM_COLS = 512;
constexpr int EPI_COLS = 8;      // accumulator columns a set drains per epilogue step
constexpr int SS_PITCH = 260;    // u32 per drained column (256 limb rows + pad, 16-byte rows)
constexpr int SS_WORDS = EPI_COLS * SS_PITCH;  // one staging buffer; two alternate per set
constexpr int SS_BYTES = 4 * SS_WORDS * 4;
constexpr int NBARS = 3 * TC_STAGES + 3;  // full, empty, acc_full/acc_empty/drain, tma
constexpr int SMEM_BYTES = TC_STAGES * STAGE_BYTES + SS_BYTES + 1024 /*align*/ + 128 /*barriers*/;
constexpr long long WAIT_CYCLES = tc::DRAIN_CYCLES;  // ~2 s at 1.9 GHz (default budget)
// instruction descriptor: D = S32 (2 << 4), A = B = U8 (0), both K-major, N = 256, M = 128
constexpr uint32_t IDESC = tc::idesc_u8(128, 256);

using tc::flag_failure;
using tc::mbar_arrive;
using tc::mbar_arrive_tx;
using tc::mbar_init;
using tc::mbar_test;
using tc::mbar_wait;
using tc::mbar_wait_drain;
using tc::mma_commit;
using tc::smem_u32;
using tc::sw128_desc;
using tc::tmem_ld16;
using tc::tmem_ld8;
using tc::tmem_wait_ld;
__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
  tc::mma_i8(dtmem, adesc, bdesc, IDESC, accumulate);
}
// All epilogue threads (barrier 1); one set's 128 threads (barriers 2 and 3).
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
__device__ __forceinline__ void set_sync(unsigned set) {
  asm volatile("bar.sync %0, 128;" ::"r"(2 + set) : "memory");
}
// Barrier of the 256 epilogue threads that also ANDs their flags, so that they leave a loop
// together (a lone warp left behind would wait at the next named barrier for good).
__device__ __forceinline__ bool epi_all(bool ok) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, 1, 256, p;\n"
      " selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)ok)
      : "memory");
  return r != 0;
}
// 16 bytes of 0/1 from bits 0-3 and 8-11, 16-19, 24-27 of x: byte k of word p is bit 8k + p.
// Applied to x and x >> 4, the 32 bits of a codeword word land in 32 K positions in the order
// alimb_kernel stores A's limb columns, two instructions per word instead of a nibble multiply
// per word.
__device__ __forceinline__ uint4 bit_spread(uint32_t x) {
  constexpr uint32_t M = 0x01010101u;
  return make_uint4(x & M, (x >> 1) & M, (x >> 2) & M, (x >> 3) & M);
}
}  // namespace

__global__ void __launch_bounds__(NTHREADS, 1)
    hash_tc_kernel(const __grid_constant__ CUtensorMap tmap_a, const u64* __restrict__ cw,
                   u64* __restrict__ H, u32* __restrict__ leaves, unsigned m, size_t two_n,
                   int* __restrict__ err, long long budget, unsigned c0, unsigned nck,
                   int mode, unsigned splits) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint32_t* Ss = (uint32_t*)(smem + TC_STAGES * STAGE_BYTES);
  uint64_t* bars = (uint64_t*)(smem + TC_STAGES * STAGE_BYTES + SS_BYTES);
  uint32_t* tmem_holder = (uint32_t*)(bars + NBARS);
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[TC_STAGES]);
  const uint32_t acc_full = smem_u32(&bars[2 * TC_STAGES]);
  const uint32_t acc_empty = smem_u32(&bars[2 * TC_STAGES + 1]);
  const uint32_t drain = smem_u32(&bars[2 * TC_STAGES + 2]);
  const uint32_t tma0 = smem_u32(&bars[2 * TC_STAGES + 3]);
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // K chunks (pairs of codeword rows) c0 .. c0 + nck - 1 of this launch; mode bit 0: add the
  // partial digest to H (else write it), bit 1: hash the leaves of the finished H.
  // Work units: (tile, split) with unit u = tile + ntiles * split; split sp sums the K chunks
  // c0 + sp nck .. c0 + sp nck + nck - 1 into its own digest slice H + sp * 32 * two_n (the
  // host sums the slices when splits > 1).  "tiles" below are units.
  const unsigned ntiles = (unsigned)(two_n / TC_N), nunits = ntiles * splits;
  const unsigned my_tiles = blockIdx.x < nunits ? (nunits - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  auto unit_tile = [&](unsigned t) { return (blockIdx.x + t * gridDim.x) % ntiles; };
  auto unit_split = [&](unsigned t) { return (blockIdx.x + t * gridDim.x) / ntiles; };
  __shared__ volatile int s_fail;

  if (tid == 0) {
    s_fail = 0;
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(full0 + 8 * s, NPROD);
      mbar_init(empty0 + 8 * s, 1);
      mbar_init(tma0 + 8 * s, 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, NEPI);
    mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_holder)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_holder;
  const unsigned nfill = my_tiles * nck;

  if (warp == 0) {
    // ---- TMA producer: A-limb tiles ----
    if (lane == 0) {
      unsigned issued = 0;
      for (unsigned f = 0; f < nfill; ++f) {
        const unsigned s = f % TC_STAGES, c = c0 + unit_split(f / nck) * nck + f % nck;
        if (f >= TC_STAGES &&
            !mbar_wait(empty0 + 8 * s, ((f / TC_STAGES) - 1) & 1, &s_fail, budget)) {
          if (!s_fail) flag_failure(&s_fail, err, 1);
          break;
        }
        const uint32_t bar = tma0 + 8 * s;
        mbar_arrive_tx(bar, A_TILE);
        const uint32_t dst = smem_u32(smem + s * STAGE_BYTES);
        const int x = (int)(c * TC_KB), y = 0;
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
            "l"((uint64_t)&tmap_a), "r"(x), "r"(y), "r"(bar)
            : "memory");
        issued = f + 1;
      }
      // Only the newest copy of each stage can still be in flight (an older one was consumed
      // before its stage was refilled): wait for those before the CTA may exit.
      for (unsigned g = issued > TC_STAGES ? issued - TC_STAGES : 0; g < issued; ++g)
        if (!mbar_wait_drain(tma0 + 8 * (g % TC_STAGES), (g / TC_STAGES) & 1)) atomicExch(err, 6);
    }
  } else if (warp == 1) {
    // ---- MMA issuer ----
    if (lane == 0) {
      unsigned f = 0;
      bool ok = true;
      for (unsigned t = 0; t < my_tiles && ok; ++t) {
        if (t > 0) {
          if (!mbar_wait(acc_empty, (t - 1) & 1, &s_fail, budget)) {
            if (!s_fail) flag_failure(&s_fail, err, 2);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
        for (unsigned c = 0; c < nck; ++c, ++f) {
          const unsigned s = f % TC_STAGES;
          if (!mbar_wait(tma0 + 8 * s, (f / TC_STAGES) & 1, &s_fail, budget) ||
              !mbar_wait(full0 + 8 * s, (f / TC_STAGES) & 1, &s_fail, budget)) {
            if (!s_fail) flag_failure(&s_fail, err, 3);
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t a_base = smem_u32(smem + s * STAGE_BYTES);
          const uint32_t b_base = a_base + A_TILE;
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int ks = 0; ks < 4; ++ks)
              mma_i8(tmem + h * 256, sw128_desc(a_base + h * (128 * TC_KB) + ks * 32),
                     sw128_desc(b_base + ks * 32), (c > 0 || ks > 0) ? 1u : 0u);
          mma_commit(empty0 + 8 * s);
        }
        if (ok) mma_commit(acc_full);
      }
      // Every MMA issued so far has completed once this arrives; wait for it before the TMEM
      // is freed (also after a failure).
      mma_commit(drain);
      if (!mbar_wait_drain(drain, 0)) atomicExch(err, 7);
    }
  } else if (warp < 6) {
    // ---- B producers (128 threads): two columns each, words loaded three fills ahead ----
    const unsigned pt = tid - 64;
    auto load_fill = [&](unsigned f, u64 (&w)[4]) {
      if (f >= nfill) return;
      const unsigned tl = f / nck, c = c0 + unit_split(tl) * nck + f % nck;
      const size_t j0 = (size_t)unit_tile(tl) * TC_N;
      const bool two = 2 * c + 1 < m;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const size_t j = j0 + pt + h * NPROD;
        w[2 * h] = __ldg(cw + (size_t)(2 * c) * two_n + j);
        w[2 * h + 1] = two ? __ldg(cw + (size_t)(2 * c + 1) * two_n + j) : 0;
      }
    };
    // one fill: wait for the stage, expand the words of fill f from w, then reuse w for the
    // loads of fill f + 3 (so each load has three stages of MMA time to arrive)
    auto fill = [&](unsigned f, u64 (&w)[4]) -> bool {
      const unsigned s = f % TC_STAGES;
      if (f >= TC_STAGES &&
          !mbar_wait(empty0 + 8 * s, ((f / TC_STAGES) - 1) & 1, &s_fail, budget)) {
        if (!s_fail) flag_failure(&s_fail, err, 4);
        return false;
      }
      uint8_t* bt = smem + s * STAGE_BYTES + A_TILE;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const unsigned j = pt + h * NPROD;
        const uint32_t x4[4] = {(uint32_t)w[2 * h], (uint32_t)(w[2 * h] >> 32),
                                (uint32_t)w[2 * h + 1], (uint32_t)(w[2 * h + 1] >> 32)};
#pragma unroll
        for (int q = 0; q < 4; ++q) {  // 32 bits -> chunks 2q, 2q + 1 (bit_spread's order)
          const uint32_t x = x4[q];
          const uint4 v0 = bit_spread(x), v1 = bit_spread(x >> 4);
          *(uint4*)(bt + j * TC_KB + (((2 * q) ^ (j & 7)) << 4)) = v0;
          *(uint4*)(bt + j * TC_KB + (((2 * q + 1) ^ (j & 7)) << 4)) = v1;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(full0 + 8 * s);
      load_fill(f + 3, w);
      return true;
    };
    u64 w0[4] = {0, 0, 0, 0}, w1[4] = {0, 0, 0, 0}, w2[4] = {0, 0, 0, 0};
    load_fill(0, w0);
    load_fill(1, w1);
    load_fill(2, w2);
    for (unsigned f = 0; f < nfill; f += 3) {
      if (!fill(f, w0)) break;
      if (f + 1 >= nfill || !fill(f + 1, w1)) break;
      if (f + 2 >= nfill || !fill(f + 2, w2)) break;
    }
  } else {
    // ---- epilogue (256 threads, warps 6-13; TMEM lane quarter = warp % 4).  Two sets of four
    // warps drain alternate 8-column steps, each through its own pair of staging buffers.
    const unsigned et = tid - (64 + NPROD), quarter = warp & 3, set = et >> 7, st_t = et & 127;
    const uint32_t lane_off = (uint32_t)(32 * quarter) << 16;
    const unsigned mrow = 32 * quarter + lane;
    for (unsigned t = 0; t < my_tiles; ++t) {
      const size_t j0 = (size_t)unit_tile(t) * TC_N;
      u64* const Hs = H + (size_t)unit_split(t) * H_ROWS * two_n;  // this split's slice
      const bool got = mbar_wait(acc_full, t & 1, &s_fail, budget);
      if (!epi_all(got)) {
        if (!s_fail) flag_failure(&s_fail, err, 5);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // The set's step k stages its columns in buffer k & 1: the step before last read that
      // buffer before the previous step's barrier, so one barrier per step suffices.
      for (int k = 0; k < TC_N / EPI_COLS / 2; ++k) {
        const unsigned q = 2 * k + set;  // column group of this step
        uint32_t* Sb = Ss + (2 * set + (k & 1)) * SS_WORDS;
        uint32_t r0[8], r1[8];
        tmem_ld8(tmem + lane_off + EPI_COLS * q, r0);
        tmem_ld8(tmem + lane_off + 256 + EPI_COLS * q, r1);
        tmem_wait_ld();
#pragma unroll
        for (int cc = 0; cc < EPI_COLS; ++cc) {
          Sb[cc * SS_PITCH + mrow] = r0[cc];
          Sb[cc * SS_PITCH + 128 + mrow] = r1[cc];
        }
        set_sync(set);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const unsigned idx = st_t + 128 * i, col = idx & (EPI_COLS - 1), r = idx >> 3;
          const uint4 lo4 = *(const uint4*)&Sb[col * SS_PITCH + 8 * r];
          const uint4 hi4 = *(const uint4*)&Sb[col * SS_PITCH + 8 * r + 4];
          const u64 a = (u64)lo4.x + ((u64)lo4.y << 8) + ((u64)lo4.z << 16) + ((u64)lo4.w << 24);
          const u64 b = (u64)hi4.x + ((u64)hi4.y << 8) + ((u64)hi4.z << 16) + ((u64)hi4.w << 24);
          const u64 lo = a + (b << 32);
          const u64 hi = (b >> 32) + (lo < a ? 1 : 0);
          u64* hp = Hs + (size_t)r * two_n + j0 + EPI_COLS * q + col;
          const u64 v = gl_reduce(lo, hi);
          *hp = (mode & 1) ? gl_add(__ldcg(hp), v) : v;
        }
      }
      // accumulators drained: the MMAs of the next tile may start
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(acc_empty);
      __threadfence_block();
      epi_sync();
      // leaf hash of each 256-byte column (C = 32 canonical u64, little-endian), from L2
      if (!(mode & 2)) continue;  // a partial digest: no leaves yet
#pragma unroll 1
      for (unsigned col = et; col < (unsigned)TC_N; col += NEPI) {
        const u64* hc = H + j0 + col;
        u32 cv[8];
        b3_init(cv);
#pragma unroll
        for (int blk = 0; blk < 4; ++blk) {
          u32 wd[16];
#pragma unroll
          for (int q2 = 0; q2 < 8; ++q2) {
            const u64 v = __ldcg(hc + (size_t)(blk * 8 + q2) * two_n);
            wd[2 * q2] = (u32)v;
            wd[2 * q2 + 1] = (u32)(v >> 32);
          }
          const u32 flags = (blk == 0 ? B3_CHUNK_START : 0) | (blk == 3 ? (B3_CHUNK_END | B3_ROOT) : 0);
          b3_compress(cv, wd, 64, flags);
        }
        uint4* lp = (uint4*)(leaves + (j0 + col) * 8);
        lp[0] = make_uint4(cv[0], cv[1], cv[2], cv[3]);
        lp[1] = make_uint4(cv[4], cv[5], cv[6], cv[7]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS)
                 : "memory");
  }
}

// ---- the int8 tensor-core peak this hash is measured against ----------------------------------
// One CTA per SM; one thread issues `iters` x 4 back-to-back tcgen05.mma.kind::i8 M128 N256 K32
// on a fixed 128 x 128-byte A tile and 256 x 128-byte B tile in shared memory (the shape and
// layout the hash uses), accumulating into TMEM; one commit at the end, waited with a bound.
constexpr int PK_SMEM = 128 * TC_KB + 256 * TC_KB + 1024 + 64;

__global__ void __launch_bounds__(128, 1) i8_peak_kernel(unsigned iters, int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bar = (uint64_t*)(smem + 128 * TC_KB + 256 * TC_KB);
  uint32_t* tmem_holder = (uint32_t*)(bar + 1);
  const unsigned tid = threadIdx.x, warp = tid >> 5;
  for (unsigned i = tid; i < (128 + 256) * TC_KB / 16; i += blockDim.x)
    ((uint4*)smem)[i] = make_uint4(0x01020304u * (i & 7), i, 0x80808080u, 0x7f7f7f7fu);
  if (tid == 0) {
    mbar_init(smem_u32(bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_holder)),
                 "r"(256)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_holder;
  if (tid == 0) {
    const uint32_t a_base = smem_u32(smem), b_base = a_base + 128 * TC_KB;
    for (unsigned i = 0; i < iters; ++i)
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        mma_i8(tmem, sw128_desc(a_base + ks * 32), sw128_desc(b_base + ks * 32),
               (i > 0 || ks > 0) ? 1u : 0u);
    mma_commit(smem_u32(bar));
    if (!mbar_wait_drain(smem_u32(bar), 0)) atomicExch(err, 8);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256)
                 : "memory");
  }
}

double i8_tensor_peak_tops(unsigned iters, int* err, cudaStream_t st) {
  int dev = 0, sms = 0;
  LGS_CUDA(cudaGetDevice(&dev));
  LGS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  LGS_CUDA(cudaFuncSetAttribute(i8_peak_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                PK_SMEM));
  cudaEvent_t e0, e1;
  LGS_CUDA(cudaEventCreate(&e0));
  LGS_CUDA(cudaEventCreate(&e1));
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {  // the first launch warms up; keep the best
    LGS_CUDA(cudaEventRecord(e0, st));
    i8_peak_kernel<<<sms, 128, PK_SMEM, st>>>(iters, err);
    LGS_LAUNCH_CHECK();
    LGS_CUDA(cudaEventRecord(e1, st));
    LGS_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    LGS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double ops = 2.0 * 128 * 256 * 32 * 4.0 * iters * sms;
    if (rep > 0 && ms > 0) best = std::max(best, ops / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

// Alimb[8r + l][kperm(k)] = byte l of A[r][k] (the 256 x W limb matrix the TMA descriptor
// covers), with the K order of the B tiles the hash's producers write: inside each aligned group
// of 32 columns, bit t of a codeword word sits at position 16 ((t >> 2) & 1) + 4 (t & 3) + (t >> 3).
__global__ void alimb_kernel(const u64* __restrict__ A, uint8_t* __restrict__ alimb, size_t W) {
  size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned r = blockIdx.y;
  if (k >= W) return;
  u64 v = A[(size_t)r * W + k];
  const unsigned t = (unsigned)(k & 31);
  const size_t kp = (k & ~(size_t)31) | (16 * ((t >> 2) & 1) + 4 * (t & 3) + (t >> 3));
#pragma unroll
  for (int l = 0; l < 8; ++l) alimb[(size_t)(r * 8 + l) * W + kp] = (uint8_t)(v >> (8 * l));
}

void alimb_from_a(const u64* A, uint8_t* alimb, size_t W, cudaStream_t st) {
  alimb_kernel<<<dim3(cdiv(W, 256), 32), 256, 0, st>>>(A, alimb, W);
  LGS_LAUNCH_CHECK();
}

// ---- host side -----------------------------------------------------------------------------
namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    LGS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess)
      throw CudaError("cuTensorMapEncodeTiled is not available from the driver");
    fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}
}  // namespace

// The TMA descriptor of the 256 x W byte matrix of A's limbs: boxes of 256 rows x 128 bytes,
// 128-byte swizzle (the K-major layout tcgen05 reads).  W must be a multiple of 64.
void make_alimb_tmap(const uint8_t* alimb, size_t W, void* tmap_out) {
  if (W % 64 || ((uintptr_t)alimb & 15)) throw ShapeError("hash: A-limb matrix misaligned");
  CUtensorMap* tm = (CUtensorMap*)tmap_out;
  cuuint64_t dims[2] = {(cuuint64_t)W, 256};
  cuuint64_t strides[1] = {(cuuint64_t)W};
  cuuint32_t box[2] = {TC_KB, 256};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)alimb, dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

// The TMA descriptor of a row-major rows x inner matrix of 64-bit integers (inner even, base
// 16-byte aligned): boxes of box_rows rows x 16 values (128 bytes), 128-byte swizzle, zeros
// outside the matrix.
void make_i64_tmap(const int64_t* base, size_t rows, size_t inner, unsigned box_rows,
                   void* tmap_out) {
  if (inner % 2 || ((uintptr_t)base & 15)) throw ShapeError("TMA: int64 matrix misaligned");
  CUtensorMap* tm = (CUtensorMap*)tmap_out;
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)inner * 8};
  cuuint32_t box[2] = {16, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(tm, CU_TENSOR_MAP_DATA_TYPE_INT64, 2, (void*)base, dims, strides, box,
                           estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

size_t tensor_map_bytes() { return sizeof(CUtensorMap); }

namespace {
// Sums the split slices of the digest (H = sum of slices, plus the old H in mode bit 0) and, in
// mode bit 1, hashes each finished column as its Merkle leaf, one thread per column.
__global__ void __launch_bounds__(256) hash_combine_kernel(const u64* __restrict__ Hp,
                                                           unsigned splits, u64* __restrict__ H,
                                                           u32* __restrict__ leaves, size_t two_n,
                                                           int mode) {
  const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= two_n) return;
  u64 v[H_ROWS];
#pragma unroll
  for (int r = 0; r < H_ROWS; ++r) {
    u64 acc = (mode & 1) ? H[(size_t)r * two_n + j] : 0;
    for (unsigned sp = 0; sp < splits; ++sp)
      acc = gl_add(acc, __ldcs(Hp + ((size_t)sp * H_ROWS + r) * two_n + j));
    H[(size_t)r * two_n + j] = acc;
    v[r] = acc;
  }
  if (!(mode & 2)) return;
  u32 cv[8];
  b3_init(cv);
#pragma unroll
  for (int blk = 0; blk < 4; ++blk) {
    u32 wd[16];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      wd[2 * q] = (u32)v[blk * 8 + q];
      wd[2 * q + 1] = (u32)(v[blk * 8 + q] >> 32);
    }
    const u32 flags = (blk == 0 ? B3_CHUNK_START : 0) | (blk == 3 ? (B3_CHUNK_END | B3_ROOT) : 0);
    b3_compress(cv, wd, 64, flags);
  }
  uint4* lp = (uint4*)(leaves + j * 8);
  lp[0] = make_uint4(cv[0], cv[1], cv[2], cv[3]);
  lp[1] = make_uint4(cv[4], cv[5], cv[6], cv[7]);
}

unsigned hash_ctas_for(unsigned max_ctas) {
  int dev = 0, sms = 0;
  LGS_CUDA(cudaGetDevice(&dev));
  LGS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return max_ctas ? std::min<unsigned>(max_ctas, (unsigned)std::max(sms, 1))
                  : (unsigned)std::max(sms, 1);
}
}  // namespace

unsigned subset_sum_hash_splits(size_t two_n, unsigned rows, unsigned max_ctas) {
  const size_t ntiles = two_n / TC_N, ctas = hash_ctas_for(max_ctas);
  const unsigned nck = (rows + 1) / 2;
  unsigned sp = 1;
  // halve the K chunks of a unit while that still leaves CTAs idle and units of >= 8 chunks
  while (ntiles * sp * 2 <= ctas && nck % (sp * 2) == 0 && nck / (sp * 2) >= 8) sp *= 2;
  return sp;
}

void subset_sum_hash_tc(const void* tmap, const u64* cw, u64* H, u32* leaves, unsigned m,
                        size_t two_n, int* err, cudaStream_t st, uint64_t wait_cycles,
                        unsigned max_ctas, unsigned row0, unsigned rows, int mode,
                        u64* split_scratch) {
  if (two_n % TC_N) throw ShapeError("hash: 2n must be a multiple of 256");
  if (m == 0 || m > 8192) throw ShapeError("hash: 1 <= m <= 8192");
  if (rows == 0) rows = m - row0;
  if (row0 % 2 || (rows % 2 && row0 + rows != m) || row0 + rows > m || mode < 0 || mode > 3)
    throw ShapeError("hash: row range must start and end on chunks of two rows");
  LGS_CUDA(cudaFuncSetAttribute(hash_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SMEM_BYTES));
  const size_t ntiles = two_n / TC_N, ctas = hash_ctas_for(max_ctas);
  const unsigned nck = (rows + 1) / 2;
  // Few column tiles (square shapes): split K over CTAs into digest slices, summed afterwards
  const unsigned splits = split_scratch ? subset_sum_hash_splits(two_n, rows, max_ctas) : 1;
  const unsigned grid = (unsigned)std::min<size_t>(ntiles * splits, ctas);
  const long long budget =
      wait_cycles ? (long long)std::min<uint64_t>(wait_cycles, (uint64_t)WAIT_CYCLES) : WAIT_CYCLES;
  if (splits == 1) {
    hash_tc_kernel<<<grid, NTHREADS, SMEM_BYTES, st>>>(*(const CUtensorMap*)tmap, cw, H, leaves,
                                                       m, two_n, err, budget, row0 / 2, nck, mode,
                                                       1u);
    LGS_LAUNCH_CHECK();
    return;
  }
  hash_tc_kernel<<<grid, NTHREADS, SMEM_BYTES, st>>>(*(const CUtensorMap*)tmap, cw, split_scratch,
                                                     leaves, m, two_n, err, budget, row0 / 2,
                                                     nck / splits, 0, splits);
  LGS_LAUNCH_CHECK();
  hash_combine_kernel<<<(unsigned)cdiv(two_n, 256), 256, 0, st>>>(split_scratch, splits, H,
                                                                 leaves, two_n, mode);
  LGS_LAUNCH_CHECK();
}

}  // namespace lgs
