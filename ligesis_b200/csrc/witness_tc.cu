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
//   warp 8     TMEM allocation and one thread issuing the MMAs (M128 N=NR K32, 6 limb pairs,
//              4 K steps per chunk) into four accumulators of NR columns
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
constexpr int WT_THREADS = WT_PROD + 32;
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

__device__ __forceinline__ void ld_pair(const int64_t* p, size_t k, size_t ke, bool row_ok,
                                        bool vec, int64_t& a, int64_t& b) {
  a = b = 0;
  if (!row_ok || k >= ke) return;
  if (vec && k + 1 < ke) {
    const longlong2 v = __ldg((const longlong2*)(p + k));
    a = v.x;
    b = v.y;
  } else {
    a = __ldg(p + k);
    if (k + 1 < ke) b = __ldg(p + k + 1);
  }
}

__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

__global__ void __launch_bounds__(WT_THREADS, 2) linear_witness_tc_kernel(const WtArgs a) {
  extern __shared__ uint8_t wt_smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)wt_smem_raw + 1023) & ~(uintptr_t)1023);
  const unsigned nr = a.nr;
  const size_t stage_bytes = wt_stage_bytes(nr);
  unsigned long long* sx = (unsigned long long*)(smem + WT_STAGES * stage_bytes);
  uint64_t* bars = (uint64_t*)(sx + WT_NR_MAX);
  uint32_t* tmem_holder = (uint32_t*)(bars + 2 * WT_STAGES + 2);
  const uint32_t full0 = tc::smem_u32(&bars[0]), empty0 = tc::smem_u32(&bars[WT_STAGES]);
  const uint32_t accf = tc::smem_u32(&bars[2 * WT_STAGES]);
  const uint32_t drain = tc::smem_u32(&bars[2 * WT_STAGES + 1]);
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
    }
    tc::mbar_init(accf, 1);
    tc::mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < WT_NR_MAX) sx[tid] = 0;
  if (warp == 8) {
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

  if (warp == 8) {
    // ---- MMA issuer: per chunk 4 K steps x 6 limb pairs; pair (i, j) into accumulator i + j
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_u8(WT_M, nr);
      bool ok = true;
      for (unsigned t = 0; t < nchunks && ok; ++t) {
        const unsigned s = t % WT_STAGES;
        if (!tc::mbar_wait(full0 + 8 * s, (t / WT_STAGES) & 1, &s_fail, a.budget)) {
          if (!s_fail) tc::flag_failure(&s_fail, a.err, 16);
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t sa = tc::smem_u32(smem + s * stage_bytes);
        const uint32_t sb = sa + (uint32_t)(WT_LW * WT_A_TILE);
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
#pragma unroll
          for (int i = 0; i < WT_LX; ++i)
#pragma unroll
            for (int j = 0; j < WT_LW; ++j) {
              // the first pair of each accumulator in the first K step overwrites it
              const bool first = t == 0 && ks == 0 && (j == 1 || i == 0) && !(i == 2 && j == 0);
              tc::mma_i8(tmem + (uint32_t)((i + j) * nr),
                         tc::sw128_desc(sa + (uint32_t)(j * WT_A_TILE) + 32 * ks),
                         tc::sw128_desc(sb + (uint32_t)(i * nr * WT_KC) + 32 * ks), idesc,
                         first ? 0u : 1u);
            }
        tc::mma_commit(empty0 + 8 * s);
      }
      if (ok) tc::mma_commit(accf);
      // every MMA issued so far has completed once this arrives: wait before the TMEM is freed
      tc::mma_commit(drain);
      if (!tc::mbar_wait_drain(drain, 0)) atomicExch(a.err, 17);
    }
  } else {
    // ---- producers: W tile (128 output columns) and X tile (nr rows) of each chunk as limbs
    bool bad = false;
    const bool wvec = a.wt && (a.inner % 2 == 0) && (((uintptr_t)a.w & 15) == 0);
    const bool xvec = (a.inner % 2 == 0) && (((uintptr_t)a.x & 15) == 0);
    for (unsigned t = 0; t < nchunks; ++t) {
      const unsigned s = t % WT_STAGES;
      if (t >= WT_STAGES &&
          !tc::mbar_wait(empty0 + 8 * s, ((t / WT_STAGES) - 1) & 1, &s_fail, a.budget)) {
        if (!s_fail) tc::flag_failure(&s_fail, a.err, 18);
        break;
      }
      uint8_t* st = smem + s * stage_bytes;
      uint8_t* const wt_tiles[WT_LW] = {st, st + WT_A_TILE};
      uint8_t* xb = st + WT_LW * WT_A_TILE;
      uint8_t* const x_tiles[WT_LX] = {xb, xb + nr * WT_KC, xb + 2 * nr * WT_KC};
      const size_t k0 = kb + (size_t)t * WT_KC;
      if (a.wt) {  // W[c][k]: warp `warp` stages rows m = 8 step + warp
#pragma unroll 4
        for (int step = 0; step < WT_M / 8; ++step) {
          const unsigned m = 8 * step + warp;
          const size_t c = c0 + m;
          const bool ok = c < a.cols;
          const int64_t* p = a.w + (ok ? c : 0) * a.inner;
          int64_t v0, v1, v2, v3;
          ld_pair(p, k0 + 2 * lane, ke, ok, wvec, v0, v1);
          ld_pair(p, k0 + 64 + 2 * lane, ke, ok, wvec, v2, v3);
          const uint32_t e0 = w_enc(v0, ok && k0 + 2 * lane < ke, bad);
          const uint32_t e1 = w_enc(v1, ok && k0 + 2 * lane + 1 < ke, bad);
          const uint32_t e2 = w_enc(v2, ok && k0 + 64 + 2 * lane < ke, bad);
          const uint32_t e3 = w_enc(v3, ok && k0 + 64 + 2 * lane + 1 < ke, bad);
          store_row<WT_LW>(wt_tiles, m, e0, e1, e2, e3);
        }
      } else {  // W[k][c]: lane = output column, four consecutive k per thread
        const unsigned m = 32 * (warp & 3) + lane;
        const size_t c = c0 + m;
        const bool ok = c < a.cols;
#pragma unroll 4
        for (int step = 0; step < WT_KC / 8; ++step) {
          const unsigned kk = 8 * step + 4 * (warp >> 2);
          uint32_t w0 = 0, w1 = 0;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const size_t k = k0 + kk + i;
            const bool valid = ok && k < ke;
            const int64_t v = valid ? __ldg(a.w + k * a.cols + c) : 0;
            const uint32_t e = w_enc(v, valid, bad);
            w0 |= (e & 255u) << (8 * i);
            w1 |= ((e >> 8) & 255u) << (8 * i);
          }
          *(uint32_t*)(wt_tiles[0] + tc::sw128_off(m, kk)) = w0;
          *(uint32_t*)(wt_tiles[1] + tc::sw128_off(m, kk)) = w1;
        }
      }
      // X tile: rows below nrv are data, row nrv is ones (limb 0), the rest zero
      for (unsigned r = warp; r < nr; r += 8) {
        const size_t gr = r0 + r;
        const bool data = r < a.nrv && gr < a.rows;
        uint32_t e0 = 0, e1 = 0, e2 = 0, e3 = 0;
        if (data) {
          const int64_t* p = a.x + gr * a.inner;
          int64_t v0, v1, v2, v3;
          ld_pair(p, k0 + 2 * lane, ke, true, xvec, v0, v1);
          ld_pair(p, k0 + 64 + 2 * lane, ke, true, xvec, v2, v3);
          e0 = x_enc(v0, k0 + 2 * lane < ke, bad);
          e1 = x_enc(v1, k0 + 2 * lane + 1 < ke, bad);
          e2 = x_enc(v2, k0 + 64 + 2 * lane < ke, bad);
          e3 = x_enc(v3, k0 + 64 + 2 * lane + 1 < ke, bad);
          const unsigned part = __reduce_add_sync(0xffffffffu, e0 + e1 + e2 + e3);
          if (lane == 0) sx[r] += part;
        } else if (r == a.nrv) {
          e0 = e1 = e2 = e3 = 1;
        }
        store_row<WT_LX>(x_tiles, r, e0, e1, e2, e3);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tc::mbar_arrive(full0 + 8 * s);
    }
    if (bad) atomicExch(a.range, 1);
    // every producer's sum of x' is in shared memory before the epilogue reads it
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
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 8) {
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
  auto k = linear_witness_tc_kernel;
  LGS_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 1, nsm = 148;
  LGS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
  LGS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, WT_THREADS, smem));
  const size_t slots = (size_t)std::max(1, per_sm) * nsm;
  const size_t mt = (cols + WT_M - 1) / WT_M, tiles = mt * ntr;
  const size_t chunks = (inner + WT_KC - 1) / WT_KC;
  // K splits: the fewest that minimise (waves of CTAs) x (chunks per CTA), and enough that no
  // CTA sums more than WT_KMAX values of K
  const size_t min_split = (inner + WT_KMAX - 1) / WT_KMAX;
  size_t split = min_split, best = SIZE_MAX;
  for (size_t sp = min_split; sp <= std::min<size_t>(chunks, 64); ++sp) {
    const size_t per = (chunks + sp - 1) / sp;
    const size_t cost = ((tiles * sp + slots - 1) / slots) * per;
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
  const dim3 grid((unsigned)mt, (unsigned)ntr, (unsigned)split);
  StageTimer t(c->prof, st, "linear_witness_tc");
  k<<<grid, WT_THREADS, smem, st>>>(a);
  LGS_LAUNCH_CHECK();
}

}  // namespace lgs
