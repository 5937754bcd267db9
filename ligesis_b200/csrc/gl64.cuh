// Goldilocks field p = 2^64 - 2^32 + 1 and its quadratic extension F_p[x]/(x^2 - 7), for host
// and device.  These are the `BF` / `EF = BinomialExtensionField<BF, 2>` of the reference prover
// (pcs/src/ligesis.rs:205-210, :787).  Values are always kept canonical (< p); an EF element is
// (c0, c1) = c0 + c1 x and is stored as two consecutive u64 (c0 first), which is also its
// serialized byte order (utils/src/merkle.rs:24-35).
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define GL_HD __host__ __device__ __forceinline__
#else
#define GL_HD inline
#endif

namespace lgs {

typedef uint64_t u64;
typedef uint32_t u32;

constexpr u64 GL_P = 0xFFFFFFFF00000001ULL;
constexpr u64 GL_EPS = 0xFFFFFFFFULL;  // 2^64 mod p
constexpr u64 GL_W = 7;                // extension non-residue
// Generator of the order-2^32 subgroup (p3-goldilocks' published value); the order-2^k
// generator is its 2^(32-k)-th power.
constexpr u64 GL_G32 = 1753635133440165772ULL;

GL_HD u64 gl_mulhi(u64 a, u64 b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (u64)(((unsigned __int128)a * b) >> 64);
#endif
}

// (hi * 2^64 + lo) mod p with 2^64 = 2^32 - 1 and 2^96 = -1.
GL_HD u64 gl_reduce(u64 lo, u64 hi) {
  u64 hh = hi >> 32, hl = hi & GL_EPS;
  u64 t0 = lo - hh;
  if (lo < hh) t0 -= GL_EPS;
  u64 t1 = (hl << 32) - hl;
  u64 t2 = t0 + t1;
  if (t2 < t1) t2 += GL_EPS;
  return t2 >= GL_P ? t2 - GL_P : t2;
}
#ifdef __CUDA_ARCH__
// Device versions on 32-bit carry chains.  Operands and results are canonical.
__device__ __forceinline__ u64 gl_pack(uint32_t lo, uint32_t hi) {
  return ((u64)hi << 32) | lo;
}
// a + b: s = a + b (carry c1), and c2 = the carry of s + eps (that is, s >= p); exactly one of
// them set means the canonical result is s + eps = s - p (mod 2^64) (a, b < p, so never both).
// The correction s + (c1 + c2) eps is one wide multiply-add, which runs on the FMA pipe instead
// of selects on the integer ALU pipe.
__device__ __forceinline__ u64 gl_add(u64 a, u64 b) {
  u64 r;
  asm("{\n\t.reg .u32 s0, s1, d, c;\n\t.reg .u64 s;\n\t"
      "add.cc.u32 s0, %1, %3;\n\t"
      "addc.cc.u32 s1, %2, %4;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "add.cc.u32 d, s0, 0xffffffff;\n\t"
      "addc.cc.u32 d, s1, 0;\n\t"
      "addc.u32 c, c, 0;\n\t"
      "mov.b64 s, {s0, s1};\n\t"
      "mad.wide.u32 %0, c, 0xffffffff, s;\n\t}"
      : "=l"(r)
      : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
  return r;
}
// a - b: on a borrow, d = a - b + 2^64 and the result is d - eps = a - b + p.
__device__ __forceinline__ u64 gl_sub(u64 a, u64 b) {
  uint32_t d0, d1;
  asm("{\n\t.reg .u32 m;\n\t"
      "sub.cc.u32 %0, %2, %4;\n\t"
      "subc.cc.u32 %1, %3, %5;\n\t"
      "subc.u32 m, 0, 0;\n\t"
      "sub.cc.u32 %0, %0, m;\n\t"
      "subc.u32 %1, %1, 0;\n\t}"
      : "=&r"(d0), "=&r"(d1)
      : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
  return gl_pack(d0, d1);
}
// (r0 + r1 2^32 + r2 2^64 + r3 2^96) mod p = (r0 + r1 2^32) - r3 + r2 (2^32 - 1).
// u = lo - r3 (minus eps on a borrow), w = u + r2 eps (plus eps on a carry, which cannot carry
// again), then the canonical w - p if w >= p.  The products and both conditional corrections
// are wide multiplies/multiply-adds (FMA pipe).
__device__ __forceinline__ u64 gl_reduce4(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
  u64 r;
  asm("{\n\t.reg .u32 u0, u1, m, v0, v1, w0, w1, d, c;\n\t.reg .u64 v, w;\n\t"
      "sub.cc.u32 u0, %1, %4;\n\t"
      "subc.cc.u32 u1, %2, 0;\n\t"
      "subc.u32 m, 0, 0;\n\t"
      "sub.cc.u32 u0, u0, m;\n\t"
      "subc.u32 u1, u1, 0;\n\t"
      "mul.wide.u32 v, %3, 0xffffffff;\n\t"
      "mov.b64 {v0, v1}, v;\n\t"
      "add.cc.u32 w0, u0, v0;\n\t"
      "addc.cc.u32 w1, u1, v1;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "mov.b64 w, {w0, w1};\n\t"
      "mad.wide.u32 w, c, 0xffffffff, w;\n\t"
      "mov.b64 {w0, w1}, w;\n\t"
      "add.cc.u32 d, w0, 0xffffffff;\n\t"
      "addc.cc.u32 d, w1, 0;\n\t"
      "addc.u32 c, 0, 0;\n\t"
      "mad.wide.u32 %0, c, 0xffffffff, w;\n\t}"
      : "=l"(r)
      : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
  return r;
}
__device__ __forceinline__ u64 gl_mul(u64 a, u64 b) {
  const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
  const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  uint32_t r0, r1, r2, r3;
  asm("mul.lo.u32 %0, %4, %6;\n\t"
      "mul.hi.u32 %1, %4, %6;\n\t"
      "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
      "madc.hi.u32 %2, %4, %7, 0;\n\t"
      "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
      "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
      "madc.hi.u32 %3, %5, %7, 0;\n\t"
      "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
      "addc.u32 %3, %3, 0;"
      : "=&r"(r0), "=&r"(r1), "=&r"(r2), "=&r"(r3)
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
  return gl_reduce4(r0, r1, r2, r3);
}
#else
GL_HD u64 gl_add(u64 a, u64 b) {
  u64 s = a + b;
  if (s < a) s += GL_EPS;
  return s >= GL_P ? s - GL_P : s;
}
GL_HD u64 gl_sub(u64 a, u64 b) { return a >= b ? a - b : a + (GL_P - b); }
GL_HD u64 gl_mul(u64 a, u64 b) { return gl_reduce(a * b, gl_mulhi(a, b)); }
#endif
GL_HD u64 gl_neg(u64 a) { return a ? GL_P - a : 0; }
#ifdef __CUDACC__
// Unreduced multiply-accumulate: acc (five 32-bit words, < 2^160) += a * b as a 128-bit product.
// Sums of up to 2^32 products are exact; gl_acc_reduce brings the sum back into the field.
struct Acc160 {
  uint32_t w[5];
};
__device__ __forceinline__ void gl_acc_zero(Acc160& a) {
  a.w[0] = a.w[1] = a.w[2] = a.w[3] = a.w[4] = 0;
}
__device__ __forceinline__ void gl_mac(Acc160& acc, u64 a, u64 b) {
#ifdef __CUDA_ARCH__
  const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
  const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  asm("{\n\t.reg .u32 r0, r1, r2, r3;\n\t"
      "mul.lo.u32 r0, %5, %7;\n\t"
      "mul.hi.u32 r1, %5, %7;\n\t"
      "mad.lo.cc.u32 r1, %5, %8, r1;\n\t"
      "madc.hi.u32 r2, %5, %8, 0;\n\t"
      "mad.lo.cc.u32 r1, %6, %7, r1;\n\t"
      "madc.hi.cc.u32 r2, %6, %7, r2;\n\t"
      "madc.hi.u32 r3, %6, %8, 0;\n\t"
      "mad.lo.cc.u32 r2, %6, %8, r2;\n\t"
      "addc.u32 r3, r3, 0;\n\t"
      "add.cc.u32 %0, %0, r0;\n\t"
      "addc.cc.u32 %1, %1, r1;\n\t"
      "addc.cc.u32 %2, %2, r2;\n\t"
      "addc.cc.u32 %3, %3, r3;\n\t"
      "addc.u32 %4, %4, 0;\n\t}"
      : "+r"(acc.w[0]), "+r"(acc.w[1]), "+r"(acc.w[2]), "+r"(acc.w[3]), "+r"(acc.w[4])
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
#endif
}
// (w0 + w1 2^32 + w2 2^64 + w3 2^96 + w4 2^128) mod p, with 2^128 = -2^32 mod p.
__device__ __forceinline__ u64 gl_acc_reduce(const Acc160& a) {
#ifdef __CUDA_ARCH__
  return gl_sub(gl_reduce4(a.w[0], a.w[1], a.w[2], a.w[3]), (u64)a.w[4] << 32);
#else
  return 0;
#endif
}
#endif
GL_HD u64 gl_canon(u64 a) { return a >= GL_P ? a - GL_P : a; }
GL_HD u64 gl_pow(u64 a, u64 e) {
  u64 r = 1;
  while (e) {
    if (e & 1) r = gl_mul(r, a);
    a = gl_mul(a, a);
    e >>= 1;
  }
  return r;
}
GL_HD u64 gl_inv(u64 a) { return gl_pow(a, GL_P - 2); }
GL_HD u64 gl_two_adic_generator(unsigned bits) {
  u64 g = GL_G32;
  for (unsigned i = bits; i < 32; ++i) g = gl_mul(g, g);
  return g;
}
// x * 2^s mod p for 0 <= s < 64.
GL_HD u64 gl_shl(u64 x, unsigned s) {
  if (s == 0) return x;
  return gl_reduce(x << s, x >> (64 - s));
}
// x * 2^s mod p for 0 <= s < 192 (2 has order 192: 2^96 = -1).  Roots of unity of order up to
// 64 are powers of two, so the small DFT butterflies multiply with shifts only.
GL_HD u64 gl_mul_pow2(u64 x, unsigned s) {
  if (s >= 96) {
    x = gl_neg(x);
    s -= 96;
  }
  if (s < 64) return gl_shl(x, s);
  // 64 <= s < 96: x = xl + 2^32 xh, 2^64 = 2^32 - 1 and 2^96 = -1 give
  // x 2^s = xl 2^(s-32) - (xl + xh) 2^(s-64): one reduction and a subtraction.
  const u64 xl = x & GL_EPS, xh = x >> 32;
  const u64 a = gl_reduce(xl << (s - 32), xl >> (96 - s));
  u64 b = (xl + xh) << (s - 64);  // < 2^64
  if (b >= GL_P) b -= GL_P;
  return gl_sub(a, b);
}
// The order-8 root the reference's generator gives: g_3 = 2^120 (checked at context creation).
constexpr unsigned GL_LOG2_OMEGA8 = 120;

struct ef2 {
  u64 c0, c1;
};
GL_HD ef2 ef_make(u64 a, u64 b) {
  ef2 r;
  r.c0 = a;
  r.c1 = b;
  return r;
}
GL_HD ef2 ef_zero() { return ef_make(0, 0); }
GL_HD ef2 ef_one() { return ef_make(1, 0); }
GL_HD ef2 ef_from(u64 a) { return ef_make(a, 0); }
GL_HD bool ef_eq(ef2 a, ef2 b) { return a.c0 == b.c0 && a.c1 == b.c1; }
GL_HD ef2 ef_add(ef2 a, ef2 b) { return ef_make(gl_add(a.c0, b.c0), gl_add(a.c1, b.c1)); }
GL_HD ef2 ef_sub(ef2 a, ef2 b) { return ef_make(gl_sub(a.c0, b.c0), gl_sub(a.c1, b.c1)); }
GL_HD ef2 ef_scale(ef2 a, u64 s) { return ef_make(gl_mul(a.c0, s), gl_mul(a.c1, s)); }
// 7 * x: x*8 - x through the 128-bit path (x < p, so x*8 < 2^67).
GL_HD u64 gl_mul7(u64 x) { return gl_sub(gl_reduce(x << 3, x >> 61), x); }
#ifdef __CUDA_ARCH__
// (w0 + w1 2^32 + w2 2^64 + w3 2^96) = a * b, the 128-bit product on 32-bit multiply-adds.
__device__ __forceinline__ void gl_mul_wide(u64 a, u64 b, uint32_t (&r)[4]) {
  const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
  const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
  asm("mul.lo.u32 %0, %4, %6;\n\t"
      "mul.hi.u32 %1, %4, %6;\n\t"
      "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
      "madc.hi.u32 %2, %4, %7, 0;\n\t"
      "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
      "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
      "madc.hi.u32 %3, %5, %7, 0;\n\t"
      "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
      "addc.u32 %3, %3, 0;"
      : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3])
      : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
}
#endif
GL_HD ef2 ef_mul(ef2 a, ef2 b) {
#ifdef __CUDA_ARCH__
  // Schoolbook with one reduction per coordinate: c1 = a0 b1 + a1 b0 and c0 = a0 b0 + 7 a1 b1 are
  // summed unreduced (below 2^129 and 2^131) in five 32-bit words, then brought into the field.
  Acc160 w1, w0;
  uint32_t t[4];
  gl_mul_wide(a.c0, b.c1, t);
  w1.w[0] = t[0], w1.w[1] = t[1], w1.w[2] = t[2], w1.w[3] = t[3], w1.w[4] = 0;
  gl_mac(w1, a.c1, b.c0);
  gl_mul_wide(a.c1, b.c1, t);  // 7 t = 8 t - t, exact in five words
  asm("{\n\t.reg .u32 s0, s1, s2, s3, s4;\n\t"
      "shl.b32 s0, %5, 3;\n\t"
      "shf.l.clamp.b32 s1, %5, %6, 3;\n\t"
      "shf.l.clamp.b32 s2, %6, %7, 3;\n\t"
      "shf.l.clamp.b32 s3, %7, %8, 3;\n\t"
      "shr.b32 s4, %8, 29;\n\t"
      "sub.cc.u32 %0, s0, %5;\n\t"
      "subc.cc.u32 %1, s1, %6;\n\t"
      "subc.cc.u32 %2, s2, %7;\n\t"
      "subc.cc.u32 %3, s3, %8;\n\t"
      "subc.u32 %4, s4, 0;\n\t}"
      : "=r"(w0.w[0]), "=r"(w0.w[1]), "=r"(w0.w[2]), "=r"(w0.w[3]), "=r"(w0.w[4])
      : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]));
  gl_mac(w0, a.c0, b.c0);
  return ef_make(gl_acc_reduce(w0), gl_acc_reduce(w1));
#else
  // Karatsuba: c0 = a0 b0 + 7 a1 b1, c1 = (a0 + a1)(b0 + b1) - a0 b0 - a1 b1
  u64 p0 = gl_mul(a.c0, b.c0), p1 = gl_mul(a.c1, b.c1);
  u64 pm = gl_mul(gl_add(a.c0, a.c1), gl_add(b.c0, b.c1));
  return ef_make(gl_add(p0, gl_mul7(p1)), gl_sub(gl_sub(pm, p0), p1));
#endif
}
// (1 - r) a + r b = a + r (b - a)
GL_HD ef2 ef_lerp(ef2 a, ef2 b, ef2 r) { return ef_add(a, ef_mul(r, ef_sub(b, a))); }
GL_HD ef2 ef_inv(ef2 a) {
  u64 norm = gl_sub(gl_mul(a.c0, a.c0), gl_mul7(gl_mul(a.c1, a.c1)));
  u64 ni = gl_inv(norm);
  return ef_make(gl_mul(a.c0, ni), gl_mul(gl_neg(a.c1), ni));
}

}  // namespace lgs
