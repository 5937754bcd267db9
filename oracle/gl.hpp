// ORACLE (test infrastructure only): a single-threaded CPU restatement of the field layer the
// reference prover uses. Only tests/, the smoke check and bench.py's CPU-baseline leg load this
// code, and only as the checker; the product library never links it.
//
// Goldilocks: p = 2^64 - 2^32 + 1 (p3-goldilocks 0.5.3, Cargo.lock:333-352; used as `BF`
// throughout pcs/src/ligesis.rs).  The quadratic extension `EF = BinomialExtensionField<BF, 2>`
// (pcs/src/ligesis.rs:787, proofsys/src/protocol.rs:7) is F_p[x]/(x^2 - W) with W = 7, the
// non-residue p3-goldilocks publishes for its degree-2 binomial extension.  Its elements are
// (c0, c1) = c0 + c1*x and serialize as c0 then c1, each as a canonical little-endian u64
// (utils/src/merkle.rs:24-35, pinned for BF by the test at utils/src/merkle.rs:147-156).
//
// Two-adic generators (p3 `TwoAdicField::two_adic_generator(bits)`, called at
// pcs/src/ligesis.rs:555, pcs/src/basefold.rs:204,223): g_32 = 1753635133440165772 generates
// the order-2^32 subgroup and g_bits = g_32^(2^(32-bits)).  The value is the one published by
// Plonky3; it is not pinned by any reference test.  tests/ check that it has order exactly 2^32
// and that g_1 = p - 1, g_2 = 2^48 (the structure every published table has).
#pragma once
#include <cstdint>
#include <cstddef>
#include <vector>
#include <stdexcept>

namespace orc {

using u64 = uint64_t;
using u128 = unsigned __int128;

constexpr u64 P = 0xFFFFFFFF00000001ULL;
constexpr u64 EPS = 0xFFFFFFFFULL;  // 2^64 mod p
constexpr u64 EXT_W = 7;            // EF non-residue
constexpr u64 G32 = 1753635133440165772ULL;

// Reduce a 128-bit integer mod p using 2^64 = 2^32 - 1 and 2^96 = -1 (mod p).
inline u64 reduce128(u128 x) {
  u64 lo = (u64)x, hi = (u64)(x >> 64);
  u64 hh = hi >> 32, hl = hi & EPS;
  u64 t0 = lo - hh;
  if (lo < hh) t0 -= EPS;  // borrow of 2^64 == -(2^32-1)
  u64 t1 = hl * EPS;       // < 2^64, exact
  u64 t2 = t0 + t1;
  if (t2 < t1) t2 += EPS;  // carry of 2^64 == 2^32-1 (cannot overflow again)
  if (t2 >= P) t2 -= P;
  return t2;
}

inline u64 canon(u64 a) { return a >= P ? a - P : a; }
inline u64 add(u64 a, u64 b) {
  u64 s = a + b;
  if (s < a) s += EPS;  // wrapped: a + b - 2^64 + (2^32 - 1)
  if (s >= P) s -= P;
  return s;
}
inline u64 sub(u64 a, u64 b) { return a >= b ? a - b : a + (P - b); }
inline u64 neg(u64 a) { return a == 0 ? 0 : P - a; }
inline u64 mul(u64 a, u64 b) { return reduce128((u128)a * b); }
inline u64 pow(u64 a, u64 e) {
  u64 r = 1;
  while (e) {
    if (e & 1) r = mul(r, a);
    a = mul(a, a);
    e >>= 1;
  }
  return r;
}
inline u64 inv(u64 a) {
  if (a == 0) throw std::runtime_error("inverse of zero");
  return pow(a, P - 2);
}
inline u64 two_adic_generator(unsigned bits) {
  if (bits > 32) throw std::runtime_error("two-adicity is 32");
  u64 g = G32;
  for (unsigned i = bits; i < 32; ++i) g = mul(g, g);
  return g;
}

struct EF {
  u64 c0 = 0, c1 = 0;
  EF() = default;
  constexpr EF(u64 a, u64 b) : c0(a), c1(b) {}
  static EF from(u64 a) { return EF(a, 0); }
  bool operator==(const EF& o) const { return c0 == o.c0 && c1 == o.c1; }
  bool operator!=(const EF& o) const { return !(*this == o); }
};
inline EF ef_zero() { return EF(0, 0); }
inline EF ef_one() { return EF(1, 0); }
inline EF operator+(EF a, EF b) { return EF(add(a.c0, b.c0), add(a.c1, b.c1)); }
inline EF operator-(EF a, EF b) { return EF(sub(a.c0, b.c0), sub(a.c1, b.c1)); }
inline EF operator*(EF a, EF b) {
  // (a0 + a1 x)(b0 + b1 x) = a0 b0 + W a1 b1 + (a0 b1 + a1 b0) x
  u64 c0 = add(mul(a.c0, b.c0), mul(EXT_W, mul(a.c1, b.c1)));
  u64 c1 = add(mul(a.c0, b.c1), mul(a.c1, b.c0));
  return EF(c0, c1);
}
inline EF operator*(EF a, u64 b) { return EF(mul(a.c0, b), mul(a.c1, b)); }
inline EF& operator+=(EF& a, EF b) { return a = a + b; }
inline EF& operator-=(EF& a, EF b) { return a = a - b; }
inline EF& operator*=(EF& a, EF b) { return a = a * b; }
inline EF ef_inv(EF a) {
  // 1/(a0 + a1 x) = (a0 - a1 x) / (a0^2 - W a1^2)
  u64 norm = sub(mul(a.c0, a.c0), mul(EXT_W, mul(a.c1, a.c1)));
  u64 ni = inv(norm);
  return EF(mul(a.c0, ni), mul(neg(a.c1), ni));
}

// Generic helpers so the protocol code can be written once for BF (u64) and EF.
inline EF lift(u64 a) { return EF(a, 0); }
inline EF lift(EF a) { return a; }

}  // namespace orc
