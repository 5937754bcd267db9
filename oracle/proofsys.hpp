// ORACLE (test infrastructure only): a single-threaded CPU restatement of proofsys' integer
// linear-layer and layer-norm witnesses (proofsys/src/tensor.rs, model.rs, witness.rs): the
// i128-accumulated matrix products, floor division with remainder by a positive constant, the
// bias row, the rounded square root of the layer norm and the lift of an i64 into Goldilocks.  Only tests/, the smoke check and bench.py's CPU-baseline leg
// load this code, and only as the checker; the product library never links it.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <initializer_list>
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

// softmax (proofsys/src/model.rs:409-443) of one n x n score matrix, causal.
inline void softmax_witness(const std::vector<i64>& sc, size_t n, const std::vector<i64>& lut,
                            i64 offset, i64 scale, i64* xm, i64* ex, i64* se, i64* pr) {
  for (size_t i = 0; i < n; ++i) {
    i64 mx = sc[i * n];
    for (size_t j = 1; j <= i; ++j) mx = std::max(mx, sc[i * n + j]);
    xm[i] = mx;
    i64 sum = 0;
    for (size_t j = 0; j < n; ++j) ex[i * n + j] = 0;
    for (size_t j = 0; j <= i; ++j) {
      const i64 idx = sc[i * n + j] - mx + offset;
      if (idx < 0 || (size_t)idx >= lut.size()) throw std::runtime_error("EXP index out of range");
      ex[i * n + j] = lut[idx];
      sum += lut[idx];
    }
    se[i] = sum;
    for (size_t j = 0; j < n; ++j)
      pr[i * n + j] = j <= i ? floor_div((i128)ex[i * n + j] * (i128)scale, (i128)sum) : 0;
  }
}

// One GPT-2 block's witness (model.rs:213-221 with layer_norm :241-279, attention :281-351, the
// softmax above and mlp :353-386).  Weight matrices are row-major: attn_w d x 3d, attn_proj_w
// d x d, fc_w d x hidden, fproj_w hidden x d.
struct BlockWeights {
  std::vector<i64> ln1_g, ln1_b, attn_w, attn_b, proj_w, proj_b, ln2_g, ln2_b, fc_w, fc_b,
      fproj_w, fproj_b;
};
struct GptDims {
  size_t n, d, heads, dh, hidden;
  i64 scale, sqrt_d_scale, offset;  // offset = max_v * scale
};
// The 36 output arrays in the order of the library's block witness (see ligesis_b200/proofsys.py).
inline std::vector<std::vector<i64>> block_witness(const std::vector<i64>& x, const GptDims& g,
                                                   const BlockWeights& w,
                                                   const std::vector<i64>& exp_lut,
                                                   const std::vector<i64>& gelu_lut) {
  const size_t n = g.n, d = g.d, H = g.heads, dh = g.dh, hid = g.hidden;
  std::vector<std::vector<i64>> out;
  auto push_ln = [&](const LayerNormWitness& l) {
    for (const std::vector<i64>* v :
         {&l.sum_x, &l.sum_x2, &l.var_sum, &l.stdv, &l.dividend, &l.quotient, &l.output})
      out.push_back(*v);
  };
  auto add = [](std::vector<i64> a, const std::vector<i64>& b) {
    for (size_t i = 0; i < a.size(); ++i) a[i] += b[i];
    return a;
  };
  // ln1, attention
  const LayerNormWitness ln1 = layer_norm_witness(x, n, d, w.ln1_g, w.ln1_b);
  push_ln(ln1);
  const LinearWitness qkv = linear_witness(ln1.output, n, d, w.attn_w, 3 * d, false, &w.attn_b,
                                           g.scale);
  std::vector<i64> scores(H * n * n), xmax(H * n), ex(H * n * n), se(H * n), prob(H * n * n),
      aoh(H * n * dh), rsc(H * n * n), raoh(H * n * dh), merged(n * d);
  for (size_t h = 0; h < H; ++h) {
    std::vector<i64> q(n * dh), k(n * dh), v(n * dh);
    for (size_t s2 = 0; s2 < n; ++s2)
      for (size_t e = 0; e < dh; ++e) {
        q[s2 * dh + e] = qkv.y[s2 * 3 * d + h * dh + e];
        k[s2 * dh + e] = qkv.y[s2 * 3 * d + d + h * dh + e];
        v[s2 * dh + e] = qkv.y[s2 * 3 * d + 2 * d + h * dh + e];
      }
    const LinearWitness sc = linear_witness(q, n, dh, k, n, true, nullptr, g.sqrt_d_scale);
    std::copy(sc.q.begin(), sc.q.end(), scores.begin() + h * n * n);
    std::copy(sc.rem.begin(), sc.rem.end(), rsc.begin() + h * n * n);
    softmax_witness(sc.q, n, exp_lut, g.offset, g.scale, &xmax[h * n], &ex[h * n * n], &se[h * n],
                    &prob[h * n * n]);
    const std::vector<i64> ph(prob.begin() + h * n * n, prob.begin() + (h + 1) * n * n);
    const LinearWitness ao = linear_witness(ph, n, n, v, dh, false, nullptr, g.scale);
    std::copy(ao.q.begin(), ao.q.end(), aoh.begin() + h * n * dh);
    std::copy(ao.rem.begin(), ao.rem.end(), raoh.begin() + h * n * dh);
    for (size_t i = 0; i < n; ++i)
      for (size_t e = 0; e < dh; ++e) merged[i * d + h * dh + e] = ao.q[i * dh + e];
  }
  const LinearWitness apr = linear_witness(merged, n, d, w.proj_w, d, false, &w.proj_b, g.scale);
  const std::vector<i64> attn_out = add(x, apr.y);
  using CV = const std::vector<i64>*;
  for (CV v : std::initializer_list<CV>{&qkv.q, &qkv.y, &scores, &xmax, &ex, &se, &prob, &aoh,
                                        &merged, &apr.q, &attn_out, &qkv.rem, &rsc, &raoh,
                                        &apr.rem})
    out.push_back(*v);
  // ln2, mlp
  const LayerNormWitness ln2 = layer_norm_witness(attn_out, n, d, w.ln2_g, w.ln2_b);
  push_ln(ln2);
  const LinearWitness fc = linear_witness(ln2.output, n, d, w.fc_w, hid, false, &w.fc_b, g.scale);
  std::vector<i64> act(n * hid);
  for (size_t i = 0; i < n * hid; ++i) {
    const i64 idx = fc.y[i] + g.offset;
    if (idx < 0 || (size_t)idx >= gelu_lut.size()) throw std::runtime_error("GELU index out of range");
    act[i] = gelu_lut[idx];
  }
  const LinearWitness fpr = linear_witness(act, n, hid, w.fproj_w, d, false, &w.fproj_b, g.scale);
  const std::vector<i64> mlp_out = add(attn_out, fpr.y);
  for (CV v : std::initializer_list<CV>{&fc.q, &fc.y, &act, &fpr.q, &mlp_out, &fc.rem, &fpr.rem})
    out.push_back(*v);
  return out;
}

}  // namespace orc
