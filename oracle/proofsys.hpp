// ORACLE (test infrastructure only): a single-threaded CPU restatement of proofsys' integer
// linear-layer and layer-norm witnesses (proofsys/src/tensor.rs, model.rs, witness.rs): the
// i128-accumulated matrix products, floor division with remainder by a positive constant, the
// bias row, the rounded square root of the layer norm and the lift of an i64 into Goldilocks.  Only tests/, the smoke check and bench.py's CPU-baseline leg
// load this code, and only as the checker; the product library never links it.
#pragma once
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "gl.hpp"

namespace orc {

using i64 = int64_t;
using i128 = __int128;

// checked_i128_to_i64 (tensor.rs:194-200)
inline i64 checked_i64(i128 x) {
  if (x < (i128)INT64_MIN || x > (i128)INT64_MAX) throw std::runtime_error("i64 overflow");
  return (i64)x;
}
// floor_div_i128 (tensor.rs:202-210)
inline i64 floor_div(i128 a, i128 b) {
  if (b <= 0) throw std::runtime_error("floor_div: divisor must be positive");
  i128 q = a / b;
  const i128 r = a % b;
  if (r < 0) q -= 1;
  return checked_i64(q);
}
// encode_i64 (witness.rs:102-108): x >= 0 -> x mod p, else -(|x| mod p)
inline u64 encode_i64(i64 x) {
  if (x >= 0) return (u64)x % P;
  const u64 m = (u64)(-(x + 1)) + 1;  // |x| without overflow at INT64_MIN
  return neg(m % P);
}

// The witness of one rescaled linear layer, `x.matmul(w)` or `x.matmul_transposed_rhs(w)`
// (tensor.rs:76-104), `.floor_div_const_with_rem(divisor)` (:121-133) and `.add_row_vector(bias)`
// (:51-60), as in proofsys/src/model.rs:360-361: q, rem and y = q + bias, row-major rows x cols.
struct LinearWitness {
  std::vector<i64> q, rem, y;
};
inline LinearWitness linear_witness(const std::vector<i64>& x, size_t rows, size_t inner,
                                    const std::vector<i64>& w, size_t cols, bool w_transposed,
                                    const std::vector<i64>* bias, i64 divisor) {
  if (x.size() != rows * inner || w.size() != inner * cols ||
      (bias && bias->size() != cols))
    throw std::runtime_error("linear_witness: shapes");
  LinearWitness out;
  out.q.resize(rows * cols);
  out.rem.resize(rows * cols);
  out.y.resize(rows * cols);
  for (size_t i = 0; i < rows; ++i)
    for (size_t j = 0; j < cols; ++j) {
      i128 acc = 0;
      for (size_t k = 0; k < inner; ++k) {
        const i64 b = w_transposed ? w[j * inner + k] : w[k * cols + j];
        acc += (i128)x[i * inner + k] * (i128)b;
      }
      const i64 v = checked_i64(acc);
      const i64 q = floor_div((i128)v, (i128)divisor);
      const i64 r = checked_i64((i128)v - (i128)q * (i128)divisor);
      const i128 y = (i128)q + (bias ? (i128)(*bias)[j] : 0);
      out.q[i * cols + j] = q;
      out.rem[i * cols + j] = r;
      out.y[i * cols + j] = checked_i64(y);
    }
  return out;
}

// round_sqrt (tensor.rs:218-222): the f64 square root rounded half away from zero.
inline i64 round_sqrt(i128 n) {
  if (n < 0) throw std::runtime_error("round_sqrt: negative");
  return checked_i64((i128)std::llround(std::sqrt((double)n)));
}

// layer_norm (proofsys/src/model.rs:241-279): per row sx, sx2, vs = d sx2 - sx^2, std =
// round_sqrt(vs + 1); per entry dividend = gain (d x - sx), quotient = floor(dividend / std),
// output = quotient + bias.
struct LayerNormWitness {
  std::vector<i64> sum_x, sum_x2, var_sum, stdv, dividend, quotient, output;
};
inline LayerNormWitness layer_norm_witness(const std::vector<i64>& x, size_t rows, size_t d,
                                           const std::vector<i64>& gain,
                                           const std::vector<i64>& bias) {
  if (x.size() != rows * d || gain.size() != d || bias.size() != d)
    throw std::runtime_error("layer_norm_witness: shapes");
  LayerNormWitness w;
  for (auto* v : {&w.sum_x, &w.sum_x2, &w.var_sum, &w.stdv}) v->resize(rows);
  for (auto* v : {&w.dividend, &w.quotient, &w.output}) v->resize(rows * d);
  const i128 dd = (i128)d;
  for (size_t r = 0; r < rows; ++r) {
    i128 sx = 0, sx2 = 0;
    for (size_t c = 0; c < d; ++c) {
      const i128 v = x[r * d + c];
      sx += v;
      sx2 += v * v;
    }
    const i128 vs = sx2 * dd - sx * sx;
    const i64 st = round_sqrt(vs + 1);
    w.sum_x[r] = checked_i64(sx);
    w.sum_x2[r] = checked_i64(sx2);
    w.var_sum[r] = checked_i64(vs);
    w.stdv[r] = st;
    for (size_t c = 0; c < d; ++c) {
      const i128 a = (i128)gain[c] * (dd * (i128)x[r * d + c] - sx);
      const i64 q = floor_div(a, (i128)st);
      w.dividend[r * d + c] = checked_i64(a);
      w.quotient[r * d + c] = q;
      w.output[r * d + c] = q + bias[c];
    }
  }
  return w;
}

}  // namespace orc
