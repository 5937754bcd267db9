// BLAKE3 for messages of at most one chunk (1024 bytes), host and device.  The reference hashes
// every Merkle leaf and every parent with `blake3::hash` (utils/src/merkle.rs:10-12, via
// rs_merkle's `concat_and_hash` for parents); every message on this path is one chunk: leaves
// are 16..1024 bytes and a parent is the 64-byte concatenation of its two children.
// The compression function follows the published BLAKE3 specification.
#pragma once
#include <cstdint>

#include "gl64.cuh"

namespace lgs {

#ifdef __CUDA_ARCH__
#define B3_ROTR(x, n) __funnelshift_r((x), (x), (n))
#else
#define B3_ROTR(x, n) (((x) >> (n)) | ((x) << (32 - (n))))
#endif

constexpr u32 B3_IV0 = 0x6A09E667u, B3_IV1 = 0xBB67AE85u, B3_IV2 = 0x3C6EF372u,
              B3_IV3 = 0xA54FF53Au, B3_IV4 = 0x510E527Fu, B3_IV5 = 0x9B05688Cu,
              B3_IV6 = 0x1F83D9ABu, B3_IV7 = 0x5BE0CD19u;
constexpr u32 B3_CHUNK_START = 1, B3_CHUNK_END = 2, B3_ROOT = 8;

#define B3_G(a, b, c, d, x, y)     \
  a = a + b + (x);                 \
  d = B3_ROTR(d ^ a, 16);          \
  c = c + d;                       \
  b = B3_ROTR(b ^ c, 12);          \
  a = a + b + (y);                 \
  d = B3_ROTR(d ^ a, 8);           \
  c = c + d;                       \
  b = B3_ROTR(b ^ c, 7);

// One round on state s with message m (already permuted for this round).
#define B3_ROUND(m)                                   \
  B3_G(s0, s4, s8, s12, m[0], m[1]);                  \
  B3_G(s1, s5, s9, s13, m[2], m[3]);                  \
  B3_G(s2, s6, s10, s14, m[4], m[5]);                 \
  B3_G(s3, s7, s11, s15, m[6], m[7]);                 \
  B3_G(s0, s5, s10, s15, m[8], m[9]);                 \
  B3_G(s1, s6, s11, s12, m[10], m[11]);               \
  B3_G(s2, s7, s8, s13, m[12], m[13]);                \
  B3_G(s3, s4, s9, s14, m[14], m[15]);

// Compress one block into the chaining value cv (8 words), counter = 0 (single chunk).
GL_HD void b3_compress(u32 cv[8], const u32 blk[16], u32 block_len, u32 flags) {
  u32 s0 = cv[0], s1 = cv[1], s2 = cv[2], s3 = cv[3], s4 = cv[4], s5 = cv[5], s6 = cv[6],
      s7 = cv[7];
  u32 s8 = B3_IV0, s9 = B3_IV1, s10 = B3_IV2, s11 = B3_IV3, s12 = 0, s13 = 0, s14 = block_len,
      s15 = flags;
  u32 m[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) m[i] = blk[i];
#pragma unroll
  for (int r = 0; r < 7; ++r) {
    B3_ROUND(m);
    if (r < 6) {
      // message permutation 2,6,3,10,7,0,4,13,1,11,12,5,9,14,15,8
      u32 t0 = m[2], t1 = m[6], t2 = m[3], t3 = m[10], t4 = m[7], t5 = m[0], t6 = m[4],
          t7 = m[13], t8 = m[1], t9 = m[11], t10 = m[12], t11 = m[5], t12 = m[9], t13 = m[14],
          t14 = m[15], t15 = m[8];
      m[0] = t0; m[1] = t1; m[2] = t2; m[3] = t3; m[4] = t4; m[5] = t5; m[6] = t6; m[7] = t7;
      m[8] = t8; m[9] = t9; m[10] = t10; m[11] = t11; m[12] = t12; m[13] = t13; m[14] = t14;
      m[15] = t15;
    }
  }
  cv[0] = s0 ^ s8; cv[1] = s1 ^ s9; cv[2] = s2 ^ s10; cv[3] = s3 ^ s11;
  cv[4] = s4 ^ s12; cv[5] = s5 ^ s13; cv[6] = s6 ^ s14; cv[7] = s7 ^ s15;
}

GL_HD void b3_init(u32 cv[8]) {
  cv[0] = B3_IV0; cv[1] = B3_IV1; cv[2] = B3_IV2; cv[3] = B3_IV3;
  cv[4] = B3_IV4; cv[5] = B3_IV5; cv[6] = B3_IV6; cv[7] = B3_IV7;
}

// Hash a message of `len` bytes (1 <= len <= 1024, len a multiple of 4 here) whose 32-bit
// little-endian words are produced by word(i).  Output: 8 words = the 32-byte digest.
template <class WordFn>
GL_HD void b3_hash_words(WordFn word, u32 len, u32 out[8]) {
  b3_init(out);
  u32 nblocks = (len + 63) / 64;
  for (u32 b = 0; b < nblocks; ++b) {
    u32 blk[16];
    u32 base = b * 16;
    u32 bl = len - b * 64 < 64 ? len - b * 64 : 64;
#pragma unroll
    for (int i = 0; i < 16; ++i) blk[i] = (u32)(i * 4) < bl ? word(base + i) : 0u;
    u32 flags = (b == 0 ? B3_CHUNK_START : 0) | (b + 1 == nblocks ? (B3_CHUNK_END | B3_ROOT) : 0);
    b3_compress(out, blk, bl, flags);
  }
}

// Parent node: hash of the 64-byte concatenation left || right.
GL_HD void b3_parent(const u32 l[8], const u32 r[8], u32 out[8]) {
  u32 blk[16];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    blk[i] = l[i];
    blk[8 + i] = r[i];
  }
  b3_init(out);
  b3_compress(out, blk, 64, B3_CHUNK_START | B3_CHUNK_END | B3_ROOT);
}

}  // namespace lgs
