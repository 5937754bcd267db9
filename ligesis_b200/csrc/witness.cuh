// Exact 128-bit accumulation and the per-output finish of proofsys' rescaled linear layer
// (proofsys/src/model.rs:360-374: Q, REM = floor_div(X W, divisor), Y = Q + bias, then
// encode_i64(Y), proofsys/src/witness.rs:102-108), shared by the CUDA-core kernel (witness.cu)
// and the tensor-core kernel (witness_tc.cu).
#pragma once
#include <cstdint>

#include "gl64.cuh"

namespace lgs {

// 128-bit accumulator as (hi:lo); a product of two i64 is added exactly.
// (two's complement in two words, added modulo 2^128 like the reference's i128)
struct Acc128 {
  uint64_t lo, hi;
};
__device__ __forceinline__ void mac128(Acc128& a, int64_t x, int64_t y) {
  const uint64_t pl = (uint64_t)x * (uint64_t)y;
  const uint64_t ph = (uint64_t)__mul64hi(x, y);
  a.lo += pl;
  a.hi += ph + (a.lo < pl ? 1 : 0);
}
__device__ __forceinline__ void add128(Acc128& a, const Acc128& b) {
  a.lo += b.lo;
  a.hi += b.hi + (a.lo < b.lo ? 1 : 0);
}
__device__ __forceinline__ bool fits_i64(uint64_t hi, uint64_t lo) {
  return (int64_t)hi == ((int64_t)lo >> 63);  // the high word extends the low word's sign
}

// Q, REM, Y, Y_field of one output from its exact sum v (in the i64 range) and its column's
// bias b; false when Q + bias leaves the i64 range.
__device__ __forceinline__ bool lw_finish_i64(int64_t v, int64_t b, int64_t d, size_t o,
                                              int64_t* q_out, int64_t* rem_out, int64_t* y_out,
                                              uint64_t* yf_out) {
  int64_t q, rm;
  if ((d & (d - 1)) == 0) {  // a power of two (the fixed-point scale): floor division is a shift
    const int sh = __ffsll(d) - 1;
    q = v >> sh;
    rm = v & (d - 1);
  } else {
    q = v / d, rm = v % d;  // floor division: a negative remainder moves q down
    if (rm < 0) {
      q -= 1;
      rm += d;
    }
  }
  const int64_t yy = (int64_t)((uint64_t)q + (uint64_t)b);
  if (((q ^ yy) & (b ^ yy)) < 0) return false;  // signed overflow of q + bias
  q_out[o] = q;
  rem_out[o] = rm;
  y_out[o] = yy;
  // encode_i64: y mod p, or -(|y| mod p).  |y| <= 2^63 < p, so no reduction is left: y itself,
  // or p - |y| (|y| >= 1 for y < 0).
  if (yf_out) yf_out[o] = yy >= 0 ? (uint64_t)yy : GL_P - ((uint64_t)(-(yy + 1)) + 1);
  return true;
}

// The same from a 128-bit sum, reading the bias of column c; false when a value leaves the i64
// range (checked_i128_to_i64 of the product, or Q + bias).
__device__ __forceinline__ bool lw_finish(const Acc128& s, const int64_t* bias, size_t c,
                                          int64_t d, size_t o, int64_t* q_out, int64_t* rem_out,
                                          int64_t* y_out, uint64_t* yf_out) {
  if (!fits_i64(s.hi, s.lo)) return false;
  return lw_finish_i64((int64_t)s.lo, bias ? bias[c] : 0, d, o, q_out, rem_out, y_out, yf_out);
}

}  // namespace lgs
