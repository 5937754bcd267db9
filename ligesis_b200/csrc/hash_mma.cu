// Subset-sum hash H = A * B (pcs/src/subset_sum.rs:43-67, called at pcs/src/ligesis.rs:302) as an
// exact 8-bit integer contraction on the tensor cores.
//
// B is never materialized: B[64 i + b][j] is bit b of the canonical RS codeword word F'[i][j]
// (pcs/src/ligesis.rs:292-299).  A's 64-bit entries are split into 8 byte limbs,
// Alimb[8 r + l][k] = byte l of A[r][k], so H[r][j] = sum_l 2^(8l) * S_l[r][j] mod p with
// S_l = Alimb_l * B an exact int32 sum (each term <= 255, at most W < 2^23 terms).
//
// This kernel issues `mma.sync.m16n8k32` (u8 x u8 -> s32).  The B fragment of that shape is
// 4 consecutive K entries per register, i.e. one nibble of a codeword word, which is expanded
// to 4 bytes with a single multiply; A limbs stream through shared memory with cp.async.
#include "kernels.cuh"

namespace lgs {

namespace {
constexpr int HM_M = 256;        // 32 digest rows x 8 limbs
constexpr int HM_N = 128;        // columns per CTA
constexpr int HM_PITCH = 80;     // bytes per A row in shared memory (64 data + 16 pad)
constexpr int HM_STAGES = 3;

__device__ __forceinline__ u32 nib_expand(u32 nib) { return (nib * 0x00204081u) & 0x01010101u; }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  u32 s = (u32)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void mma_u8(int* c, const u32* a, u32 b0, u32 b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// (S << 8l) mod p for a non-negative 31-bit limb sum S.
__device__ __forceinline__ u64 limb_term(u32 s, unsigned l) {
  unsigned sh = 8 * l;
  u64 lo = (u64)s << sh;
  u64 hi = sh ? ((u64)s >> (64 - sh)) : 0;
  return gl_reduce(lo, hi);
}
}  // namespace

// grid.x = two_n / 128.  256 threads: warp w -> rows 64*(w&3).., columns 64*(w>>2)..
__global__ void __launch_bounds__(256, 1)
    hash_mma_kernel(const uint8_t* __restrict__ alimb, const u64* __restrict__ cw,
                    u64* __restrict__ H, unsigned m, size_t two_n) {
  extern __shared__ __align__(16) uint8_t smem[];
  const unsigned W = 64 * m;
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned g = lane >> 2, tig = lane & 3;
  const unsigned wm = warp & 3, wn = warp >> 2;
  const size_t j0 = (size_t)blockIdx.x * HM_N + wn * 64;

  auto load_stage = [&](unsigned i, int stage) {
    uint8_t* dst = smem + stage * (HM_M * HM_PITCH);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      unsigned idx = tid + q * 256;  // 1024 16-byte pieces
      unsigned row = idx >> 2, ch = idx & 3;
      cp_async16(dst + row * HM_PITCH + ch * 16, alimb + (size_t)row * W + (size_t)i * 64 + ch * 16);
    }
  };

  int acc[4][8][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0;

#pragma unroll
  for (int s = 0; s < HM_STAGES - 1; ++s) {
    if ((unsigned)s < m) load_stage(s, s);
    cp_async_commit();
  }

  for (unsigned i = 0; i < m; ++i) {
    cp_async_wait<HM_STAGES - 2>();
    __syncthreads();
    {
      unsigned nx = i + HM_STAGES - 1;
      if (nx < m) load_stage(nx, nx % HM_STAGES);
      cp_async_commit();
    }
    const uint8_t* As = smem + (i % HM_STAGES) * (HM_M * HM_PITCH);
    u64 words[8];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) words[nt] = __ldg(cw + (size_t)i * two_n + j0 + nt * 8 + g);
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) {
      u32 a[4][4];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const uint8_t* base = As + (wm * 64 + mt * 16 + g) * HM_PITCH + kk * 32 + tig * 4;
        a[mt][0] = *(const u32*)(base);
        a[mt][1] = *(const u32*)(base + 8 * HM_PITCH);
        a[mt][2] = *(const u32*)(base + 16);
        a[mt][3] = *(const u32*)(base + 8 * HM_PITCH + 16);
      }
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        u32 half = kk ? (u32)(words[nt] >> 32) : (u32)words[nt];
        u32 b0 = nib_expand((half >> (4 * tig)) & 15u);
        u32 b1 = nib_expand((half >> (16 + 4 * tig)) & 15u);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) mma_u8(acc[mt][nt], a[mt], b0, b1);
      }
    }
  }
  cp_async_wait<0>();

  // Epilogue: lanes sharing tig hold limbs l = g of the same (r, column); combine over g.
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        u64 t = limb_term((u32)acc[mt][nt][c], g);
#pragma unroll
        for (int x = 4; x <= 16; x <<= 1) t = gl_add(t, __shfl_xor_sync(0xffffffffu, t, x));
        if (g == (unsigned)c) {  // spread the 4 stores over 4 lanes
          unsigned r = wm * 8 + mt * 2 + (c >> 1);
          size_t col = j0 + nt * 8 + tig * 2 + (c & 1);
          H[(size_t)r * two_n + col] = t;
        }
      }
}

void alimb_from_a(const u64* A, uint8_t* alimb, size_t W, cudaStream_t st);

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

void subset_sum_hash(const uint8_t* alimb, const u64* cw, u64* H, unsigned m, size_t two_n,
                     cudaStream_t st) {
  if (two_n % HM_N) throw ShapeError("hash: 2n must be a multiple of 128");
  size_t smem = (size_t)HM_STAGES * HM_M * HM_PITCH;
  static int attr_dev = -1;
  int dev;
  LGS_CUDA(cudaGetDevice(&dev));
  if (attr_dev != dev) {
    LGS_CUDA(cudaFuncSetAttribute(hash_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    attr_dev = dev;
  }
  hash_mma_kernel<<<(unsigned)(two_n / HM_N), 256, smem, st>>>(alimb, cw, H, m, two_n);
  LGS_LAUNCH_CHECK();
}

}  // namespace lgs
