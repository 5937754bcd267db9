// Subset-sum hash H = A * B (pcs/src/subset_sum.rs:43-67, called at pcs/src/ligesis.rs:302) on
// the 5th-generation tensor cores, fused with the Merkle leaf hashes of H's columns
// (pcs/src/ligesis.rs:306-313).
//
// Exactness: A's canonical 64-bit entries are split into byte limbs, Alimb[8r + l][k] = byte l of
// A[r][k], and B[64 i + b][j] = bit b of the RS codeword word F'[i][j].  S_l = Alimb_l * B is an
// exact int32 sum (terms <= 255, at most 64 * 2^13 of them), and H[r][j] = sum_l 2^(8l) S_l mod p
// is recombined exactly in 128-bit arithmetic.
//
// CTA tile: all 256 limb rows (two M = 128 accumulators in TMEM, 2 x 256 columns = the SM's
// 512 TMEM columns) by 256 codeword columns (N = 256); K advances 128 bytes (two codeword rows)
// per pipeline stage, 3 stages.
//   warp 5        TMA producer: the 256 x 128-byte A-limb tile, SWIZZLE_128B, no multicast
//   warps 0-3     B producers: expand 2 x 256 codeword words into the 256 x 128-byte K-major
//                 SWIZZLE_128B bit tile; later the epilogue
//   warp 4        TMEM allocation, and one thread issuing tcgen05.mma.kind::i8 (M128 N256 K32)
// Epilogue: tcgen05.ld the int32 limb sums, recombine mod p, write H, hash each 256-byte column
// leaf with BLAKE3 into the Merkle tree's leaf layer.  Every mbarrier wait is bounded by a clock
// budget; on timeout the CTA records an error code, stops issuing work, waits (bounded) for its
// issued MMAs, frees its TMEM and exits.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "blake3.cuh"
#include "kernels.cuh"

namespace lgs {

namespace {
constexpr int TC_N = 256;
constexpr int TC_KB = 128;
constexpr int TC_STAGES = 3;
constexpr int A_TILE = 256 * TC_KB;
constexpr int B_TILE = TC_N * TC_KB;
constexpr int STAGE_BYTES = A_TILE + B_TILE;
constexpr int NPROD = 128;
constexpr int NTHREADS = 192;
constexpr int TMEM_COLS = 512;
constexpr int SMEM_BYTES = TC_STAGES * STAGE_BYTES + 1024 /*align*/ + 128 /*barriers*/;
constexpr long long WAIT_CYCLES = 4000000000LL;  // ~2 s at 1.9 GHz
// instruction descriptor: D = S32 (2 << 4), A = B = U8 (0), both K-major, N = 256, M = 128
constexpr uint32_t IDESC = (2u << 4) | ((256u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
// Bounded wait for the phase with the given parity to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > WAIT_CYCLES) return false;
  }
}
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)1 << 16;                          // leading byte offset (unused: K fits the atom)
  d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset: 8 rows x 128 B
  d |= (uint64_t)1 << 46;                          // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                          // SWIZZLE_128B
  return d;
}
__device__ __forceinline__ void mma_i8(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t nib_expand(uint32_t nib) {
  return (nib * 0x00204081u) & 0x01010101u;
}
}  // namespace

__global__ void __launch_bounds__(NTHREADS, 1)
    hash_tc_kernel(const __grid_constant__ CUtensorMap tmap_a, const u64* __restrict__ cw,
                   u64* __restrict__ H, u32* __restrict__ leaves, unsigned m, size_t two_n,
                   int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* bars = (uint64_t*)(smem + TC_STAGES * STAGE_BYTES);
  uint32_t* tmem_holder = (uint32_t*)(bars + 8);
  const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[3]), done = smem_u32(&bars[6]);
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t j0 = (size_t)blockIdx.x * TC_N;
  const unsigned nchunks = (m + 1) / 2;
  __shared__ int s_fail;

  if (tid == 0) {
    s_fail = 0;
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(full0 + 8 * s, NPROD + 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 4) {
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

  if (warp == 5) {
    // ---- TMA producer: A-limb tiles ----
    if (lane == 0) {
      for (unsigned c = 0; c < nchunks; ++c) {
        const unsigned s = c % TC_STAGES;
        if (c >= TC_STAGES && !mbar_wait(empty0 + 8 * s, ((c / TC_STAGES) - 1) & 1)) {
          atomicExch(err, 1);
          s_fail = 1;
          break;
        }
        if (s_fail) break;
        const uint32_t bar = full0 + 8 * s;
        mbar_arrive_tx(bar, A_TILE);
        const uint32_t dst = smem_u32(smem + s * STAGE_BYTES);
        const int x = (int)(c * TC_KB), y = 0;
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
            "l"((uint64_t)&tmap_a), "r"(x), "r"(y), "r"(bar)
            : "memory");
      }
    }
  } else if (warp == 4) {
    // ---- MMA issuer ----
    if (lane == 0) {
      bool ok = true;
      for (unsigned c = 0; c < nchunks && ok; ++c) {
        const unsigned s = c % TC_STAGES;
        if (!mbar_wait(full0 + 8 * s, (c / TC_STAGES) & 1)) {
          atomicExch(err, 2);
          s_fail = 1;
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a_base = smem_u32(smem + s * STAGE_BYTES);
        const uint32_t b_base = a_base + A_TILE;
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
            mma_i8(tmem + t * 256, sw128_desc(a_base + t * (128 * TC_KB) + ks * 32),
                   sw128_desc(b_base + ks * 32), (c > 0 || ks > 0) ? 1u : 0u);
        mma_commit(empty0 + 8 * s);
      }
      mma_commit(done);  // arrives once every issued MMA has completed
    }
  } else {
    // ---- B producers (threads 0..127) ----
    for (unsigned c = 0; c < nchunks; ++c) {
      const unsigned s = c % TC_STAGES;
      if (c >= TC_STAGES && !mbar_wait(empty0 + 8 * s, ((c / TC_STAGES) - 1) & 1)) {
        atomicExch(err, 3);
        s_fail = 1;
        break;
      }
      if (s_fail) break;
      uint8_t* bt = smem + s * STAGE_BYTES + A_TILE;
      for (unsigned j = tid; j < TC_N; j += NPROD) {
        const u64 w0 = __ldg(cw + (size_t)(2 * c) * two_n + j0 + j);
        const u64 w1 = (2 * c + 1 < m) ? __ldg(cw + (size_t)(2 * c + 1) * two_n + j0 + j) : 0;
#pragma unroll
        for (int kc = 0; kc < 8; ++kc) {
          const uint32_t b16 = (uint32_t)((kc < 4 ? (w0 >> (16 * kc)) : (w1 >> (16 * (kc - 4)))) & 0xFFFFu);
          uint4 v;
          v.x = nib_expand(b16 & 15u);
          v.y = nib_expand((b16 >> 4) & 15u);
          v.z = nib_expand((b16 >> 8) & 15u);
          v.w = nib_expand((b16 >> 12) & 15u);
          *(uint4*)(bt + j * TC_KB + ((kc ^ (j & 7)) << 4)) = v;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(full0 + 8 * s);
    }
  }

  // ---- epilogue (warps 0-3) ----
  if (warp < 4) {
    const bool got = mbar_wait(done, 0);
    if (!got) atomicExch(err, 4);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    uint32_t* Ss = (uint32_t*)smem;                    // [32 cols][256 limb rows]
    u64* Hs = (u64*)(smem + 32 * 256 * 4);             // [256 cols][33] (padded)
    for (int q = 0; q < TC_N / 32; ++q) {
      uint32_t r0[32], r1[32];
      const uint32_t lane_off = (uint32_t)(32 * warp) << 16;
      tmem_ld32(tmem + lane_off + 32 * q, r0);
      tmem_ld32(tmem + lane_off + 256 + 32 * q, r1);
      const unsigned mrow = 32 * warp + lane;
#pragma unroll
      for (int cc = 0; cc < 32; ++cc) {
        Ss[cc * 256 + mrow] = r0[cc];
        Ss[cc * 256 + 128 + mrow] = r1[cc];
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const unsigned idx = tid + 128 * i, r = idx & 31, col = idx >> 5;
        const uint4 lo4 = *(const uint4*)&Ss[col * 256 + 8 * r];
        const uint4 hi4 = *(const uint4*)&Ss[col * 256 + 8 * r + 4];
        const u64 a = (u64)lo4.x + ((u64)lo4.y << 8) + ((u64)lo4.z << 16) + ((u64)lo4.w << 24);
        const u64 b = (u64)hi4.x + ((u64)hi4.y << 8) + ((u64)hi4.z << 16) + ((u64)hi4.w << 24);
        const u64 lo = a + (b << 32);
        const u64 hi = (b >> 32) + (lo < a ? 1 : 0);
        Hs[(32 * q + col) * 33 + r] = gl_reduce(lo, hi);
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
    }
    // H to global (row-major 32 x two_n), coalesced along columns
    for (unsigned r = 0; r < 32; ++r)
      for (unsigned col = tid; col < (unsigned)TC_N; col += NPROD)
        H[(size_t)r * two_n + j0 + col] = Hs[col * 33 + r];
    // leaf hash of each 256-byte column (C = 32 canonical u64, little-endian)
    for (unsigned col = tid; col < (unsigned)TC_N; col += NPROD) {
      const u64* hc = Hs + col * 33;
      u32 cv[8];
      b3_init(cv);
#pragma unroll
      for (int blk = 0; blk < 4; ++blk) {
        u32 w[16];
#pragma unroll
        for (int q2 = 0; q2 < 8; ++q2) {
          const u64 v = hc[blk * 8 + q2];
          w[2 * q2] = (u32)v;
          w[2 * q2 + 1] = (u32)(v >> 32);
        }
        const u32 flags = (blk == 0 ? B3_CHUNK_START : 0) | (blk == 3 ? (B3_CHUNK_END | B3_ROOT) : 0);
        b3_compress(cv, w, 64, flags);
      }
#pragma unroll
      for (int q2 = 0; q2 < 8; ++q2) leaves[(j0 + col) * 8 + q2] = cv[q2];
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 4) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS)
                 : "memory");
  }
}

// Alimb[8r + l][k] = byte l of A[r][k] (the 256 x W limb matrix the TMA descriptor covers).
__global__ void alimb_kernel(const u64* __restrict__ A, uint8_t* __restrict__ alimb, size_t W) {
  size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned r = blockIdx.y;
  if (k >= W) return;
  u64 v = A[(size_t)r * W + k];
#pragma unroll
  for (int l = 0; l < 8; ++l) alimb[(size_t)(r * 8 + l) * W + k] = (uint8_t)(v >> (8 * l));
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
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

size_t tensor_map_bytes() { return sizeof(CUtensorMap); }

void subset_sum_hash_tc(const void* tmap, const u64* cw, u64* H, u32* leaves, unsigned m,
                        size_t two_n, int* err, cudaStream_t st) {
  if (two_n % TC_N) throw ShapeError("hash: 2n must be a multiple of 256");
  if (m == 0 || m > 8192) throw ShapeError("hash: 1 <= m <= 8192");
  LGS_CUDA(cudaFuncSetAttribute(hash_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                SMEM_BYTES));
  hash_tc_kernel<<<(unsigned)(two_n / TC_N), NTHREADS, SMEM_BYTES, st>>>(
      *(const CUtensorMap*)tmap, cw, H, leaves, m, two_n, err);
  LGS_LAUNCH_CHECK();
}

}  // namespace lgs
