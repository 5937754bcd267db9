// ORACLE (test infrastructure only): BLAKE3 (blake3 1.8.5, Cargo.lock:36; called as
// `blake3::hash` at utils/src/merkle.rs:10-12) restated from the published BLAKE3 specification:
// 7-round compression over a 16-word state, 1024-byte chunks of 64-byte blocks, and a binary
// tree of chunk chaining values.  Only the unkeyed 32-byte `hash` mode is needed.  The
// implementation is checked against the `blake3` Python package on a range of input lengths
// (tests/golden/make_golden.py writes those known answers).
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>

namespace orc {

struct Blake3 {
  static constexpr uint32_t IV[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                     0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};
  static constexpr int PERM[16] = {2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8};
  enum : uint32_t { CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8 };

  static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
  static void g(uint32_t* s, int a, int b, int c, int d, uint32_t x, uint32_t y) {
    s[a] = s[a] + s[b] + x;
    s[d] = rotr(s[d] ^ s[a], 16);
    s[c] = s[c] + s[d];
    s[b] = rotr(s[b] ^ s[c], 12);
    s[a] = s[a] + s[b] + y;
    s[d] = rotr(s[d] ^ s[a], 8);
    s[c] = s[c] + s[d];
    s[b] = rotr(s[b] ^ s[c], 7);
  }
  // Full 16-word compression output.
  static void compress(const uint32_t cv[8], const uint32_t block[16], uint64_t counter,
                       uint32_t block_len, uint32_t flags, uint32_t out[16]) {
    uint32_t s[16] = {cv[0], cv[1], cv[2], cv[3], cv[4], cv[5], cv[6], cv[7],
                      IV[0], IV[1], IV[2], IV[3], (uint32_t)counter, (uint32_t)(counter >> 32),
                      block_len, flags};
    uint32_t m[16];
    std::memcpy(m, block, 64);
    for (int r = 0; r < 7; ++r) {
      g(s, 0, 4, 8, 12, m[0], m[1]);
      g(s, 1, 5, 9, 13, m[2], m[3]);
      g(s, 2, 6, 10, 14, m[4], m[5]);
      g(s, 3, 7, 11, 15, m[6], m[7]);
      g(s, 0, 5, 10, 15, m[8], m[9]);
      g(s, 1, 6, 11, 12, m[10], m[11]);
      g(s, 2, 7, 8, 13, m[12], m[13]);
      g(s, 3, 4, 9, 14, m[14], m[15]);
      if (r < 6) {
        uint32_t t[16];
        for (int i = 0; i < 16; ++i) t[i] = m[PERM[i]];
        std::memcpy(m, t, 64);
      }
    }
    for (int i = 0; i < 8; ++i) {
      out[i] = s[i] ^ s[i + 8];
      out[i + 8] = s[i + 8] ^ cv[i];
    }
  }
  static void load_block(const uint8_t* p, size_t len, uint32_t w[16]) {
    uint8_t buf[64] = {0};
    std::memcpy(buf, p, len);
    for (int i = 0; i < 16; ++i)
      w[i] = (uint32_t)buf[4 * i] | ((uint32_t)buf[4 * i + 1] << 8) |
             ((uint32_t)buf[4 * i + 2] << 16) | ((uint32_t)buf[4 * i + 3] << 24);
  }
  // Chaining value (or root output when is_root) of one chunk of <= 1024 bytes.
  static void chunk_cv(const uint8_t* p, size_t len, uint64_t chunk_idx, bool is_root,
                       uint32_t cv_out[8]) {
    uint32_t cv[8];
    std::memcpy(cv, IV, 32);
    size_t nblocks = len == 0 ? 1 : (len + 63) / 64;
    for (size_t b = 0; b < nblocks; ++b) {
      size_t off = b * 64;
      size_t bl = len - off < 64 ? len - off : 64;
      if (len == 0) bl = 0;
      uint32_t w[16];
      load_block(p + off, bl, w);
      uint32_t flags = 0;
      if (b == 0) flags |= CHUNK_START;
      if (b + 1 == nblocks) flags |= CHUNK_END | (is_root ? ROOT : 0);
      uint32_t out[16];
      compress(cv, w, chunk_idx, (uint32_t)bl, flags, out);
      std::memcpy(cv, out, 32);
    }
    std::memcpy(cv_out, cv, 32);
  }
  static void parent_cv(const uint32_t l[8], const uint32_t r[8], bool is_root,
                        uint32_t out_cv[8]) {
    uint32_t block[16];
    std::memcpy(block, l, 32);
    std::memcpy(block + 8, r, 32);
    uint32_t out[16];
    compress(IV, block, 0, 64, PARENT | (is_root ? ROOT : 0), out);
    std::memcpy(out_cv, out, 32);
  }
  // Root chaining value of chunks [first, first+count) (count >= 1); `root` marks the top call.
  static void subtree(const uint8_t* data, size_t len, uint64_t first, uint64_t count,
                      bool root, uint32_t cv[8]) {
    if (count == 1) {
      size_t off = first * 1024;
      size_t cl = len - off < 1024 ? len - off : 1024;
      chunk_cv(data + off, cl, first, root, cv);
      return;
    }
    uint64_t left = 1;
    while (left * 2 < count) left *= 2;  // largest power of two strictly below count
    uint32_t l[8], r[8];
    subtree(data, len, first, left, false, l);
    subtree(data, len, first + left, count - left, false, r);
    parent_cv(l, r, root, cv);
  }
  static void hash(const uint8_t* data, size_t len, uint8_t out[32]) {
    uint64_t chunks = len == 0 ? 1 : (len + 1023) / 1024;
    uint32_t cv[8];
    subtree(data, len, 0, chunks, true, cv);
    for (int i = 0; i < 8; ++i) {
      out[4 * i] = (uint8_t)cv[i];
      out[4 * i + 1] = (uint8_t)(cv[i] >> 8);
      out[4 * i + 2] = (uint8_t)(cv[i] >> 16);
      out[4 * i + 3] = (uint8_t)(cv[i] >> 24);
    }
  }
};

}  // namespace orc
