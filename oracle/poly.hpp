// ORACLE (test infrastructure only): MlPoly (utils/src/poly.rs:4-61), the product sumcheck
// (utils/src/sumcheck.rs:37-130), the radix-2 DFT the reference takes from p3-dft 0.5.3
// (`Radix2Dit::dft` / `dft_algebra`, Cargo.lock:318; call sites pcs/src/ligesis.rs:225-235,
// pcs/src/basefold.rs:346-379) and the pre-drawn randomness oracle (utils/src/oracle.rs:10-64).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "gl.hpp"
#include "par.hpp"

namespace orc {

// ---- MlPoly (utils/src/poly.rs) -----------------------------------------------------------
// eval binds the LOW variable first: s[i] = s[2i] + (s[2i+1] - s[2i]) * r   (poly.rs:7-18).
inline EF mle_eval(std::vector<EF> s, const std::vector<EF>& point) {
  if ((size_t(1) << point.size()) != s.size()) throw std::runtime_error("mle_eval size");
  size_t cur = s.size() >> 1;
  std::vector<EF> nx(cur);
  for (const EF& r : point) {
    parallel_ranges(cur, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; ++i) nx[i] = s[2 * i] + (s[2 * i + 1] - s[2 * i]) * r;
    }, size_t(1) << 15);
    std::copy(nx.begin(), nx.begin() + cur, s.begin());
    cur >>= 1;
  }
  return s[0];
}
// fold: the same recurrence for the first |point| variables, then truncate (poly.rs:33-42).
inline void mle_fold(std::vector<EF>& s, const std::vector<EF>& point) {
  size_t cur = s.size();
  for (const EF& r : point) {
    cur >>= 1;
    for (size_t i = 0; i < cur; ++i) s[i] = s[2 * i] + (s[2 * i + 1] - s[2 * i]) * r;
  }
  s.resize(cur);
}
// new_eq iterates point.rev(), so point[0] ends up on the lowest index bit (poly.rs:44-53).
inline std::vector<EF> new_eq(const std::vector<EF>& point) {
  std::vector<EF> ev{ef_one()};
  for (size_t t = point.size(); t-- > 0;) {
    const EF& p = point[t];
    std::vector<EF> nx(ev.size() * 2);
    parallel_ranges(ev.size(), [&](size_t lo, size_t hi) {
      for (size_t j = lo; j < hi; ++j) {
        nx[2 * j] = (ef_one() - p) * ev[j];
        nx[2 * j + 1] = p * ev[j];
      }
    }, size_t(1) << 15);
    ev.swap(nx);
  }
  return ev;
}
inline EF eval_eq(const std::vector<EF>& a, const std::vector<EF>& b) {  // poly.rs:55-61
  EF res = ef_one();
  size_t n = a.size() < b.size() ? a.size() : b.size();
  for (size_t i = 0; i < n; ++i) res *= a[i] * b[i] + (ef_one() - a[i]) * (ef_one() - b[i]);
  return res;
}
// split(n): num_chunks = len/n; chunk j collects elements j, j+num_chunks, ... (poly.rs:20-31).
template <class T>
inline std::vector<std::vector<T>> mle_split(const std::vector<T>& v, size_t n) {
  size_t num_chunks = v.size() / n;
  std::vector<std::vector<T>> out(num_chunks);
  for (size_t i = 0; i < v.size(); i += num_chunks)
    for (size_t j = 0; j < num_chunks; ++j) out[j].push_back(v[i + j]);
  return out;
}

// ---- radix-2 DFT: out[j] = sum_k c_k g^(jk), g = two_adic_generator(log N), natural order ----
inline void dft_bf(std::vector<u64>& a) {
  size_t n = a.size();
  unsigned logn = 0;
  while ((size_t(1) << logn) < n) ++logn;
  if ((size_t(1) << logn) != n) throw std::runtime_error("dft size");
  for (size_t i = 1, j = 0; i < n; ++i) {  // bit-reversal permutation
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (unsigned s = 1; s <= logn; ++s) {
    size_t len = size_t(1) << s, half = len >> 1;
    u64 w_len = two_adic_generator(s);
    std::vector<u64> tw(half);
    tw[0] = 1;
    for (size_t k = 1; k < half; ++k) tw[k] = mul(tw[k - 1], w_len);
    parallel_ranges(n / 2, [&](size_t lo, size_t hi) {
      for (size_t t = lo; t < hi; ++t) {
        size_t i = (t >> (s - 1)) << s, k = t & (half - 1);
        u64 u = a[i + k], v = mul(a[i + k + half], tw[k]);
        a[i + k] = add(u, v);
        a[i + k + half] = sub(u, v);
      }
    }, size_t(1) << 15);
  }
}
// dft_algebra over EF: the base-field DFT applied coordinate-wise.
inline void dft_ef(std::vector<EF>& a) {
  std::vector<u64> x(a.size()), y(a.size());
  for (size_t i = 0; i < a.size(); ++i) x[i] = a[i].c0, y[i] = a[i].c1;
  dft_bf(x);
  dft_bf(y);
  for (size_t i = 0; i < a.size(); ++i) a[i] = EF(x[i], y[i]);
}

// ---- RandomOracle (utils/src/oracle.rs:10-64): two pre-drawn arrays read by cursors ---------
struct Oracle {
  const EF* fields = nullptr;
  size_t nfields = 0;
  const u64* ints = nullptr;
  size_t nints = 0;
  size_t fi = 0, ii = 0;
  EF next_field() {
    if (fi >= nfields) throw std::runtime_error("oracle exhausted (fields)");
    return fields[fi++];
  }
  std::vector<EF> next_n_fields(size_t n) {
    std::vector<EF> v;
    for (size_t i = 0; i < n; ++i) v.push_back(next_field());
    return v;
  }
  u64 next_int() {
    if (ii >= nints) throw std::runtime_error("oracle exhausted (ints)");
    return ints[ii++];
  }
  std::vector<u64> next_n_ints(size_t n) {
    std::vector<u64> v;
    for (size_t i = 0; i < n; ++i) v.push_back(next_int());
    return v;
  }
  void restart() { fi = ii = 0; }
};

// ---- product sumcheck (utils/src/sumcheck.rs:8-130) ------------------------------------------
struct SumcheckProof {
  std::vector<std::vector<EF>> round_polys;  // each d+1 evaluations at t = 0..d
  std::vector<EF> final_evals;
};

// Binds the HIGH variable first (lo = i, hi = i + half) (sumcheck.rs:52-73).
inline SumcheckProof sumcheck_prove(std::vector<std::vector<EF>> polys, Oracle& o,
                                    std::vector<EF>* challenges) {
  if (polys.empty()) throw std::runtime_error("sumcheck: no polys");
  size_t d = polys.size();
  size_t len = polys[0].size();
  unsigned n = 0;
  while ((size_t(1) << n) < len) ++n;
  SumcheckProof pf;
  challenges->clear();
  for (unsigned round = 0; round < n; ++round) {
    size_t half = polys[0].size() / 2;
    // Per-range partial sums, added afterwards: the residues are exact, so the split
    // does not change the round polynomial.
    const size_t grain = size_t(1) << 14;
    std::vector<std::vector<EF>> part(parallel_parts(half, grain), std::vector<EF>(d + 1, ef_zero()));
    parallel_chunks(half, grain, [&](size_t pi, size_t lo, size_t hi) {
      auto& ev = part[pi];
      for (size_t i = lo; i < hi; ++i) {
        for (size_t k = 0; k <= d; ++k) {
          EF t = EF::from(k);
          EF prod = ef_one();
          for (auto& p : polys) prod *= p[i] + t * (p[i + half] - p[i]);
          ev[k] += prod;
        }
      }
    });
    std::vector<EF> evals(d + 1, ef_zero());
    for (auto& ev : part)
      for (size_t k = 0; k <= d; ++k) evals[k] += ev[k];
    pf.round_polys.push_back(evals);
    EF r = o.next_field();
    challenges->push_back(r);
    for (auto& p : polys) {
      parallel_ranges(half, [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) p[i] = p[i] + r * (p[i + half] - p[i]);
      }, grain);
      p.resize(half);
    }
  }
  for (auto& p : polys) pf.final_evals.push_back(p[0]);
  return pf;
}

// Lagrange through (0, e0) .. (d, ed), evaluated at r (sumcheck.rs:88-103).
inline EF interpolate(const std::vector<EF>& evals, EF r) {
  EF acc = ef_zero();
  size_t m = evals.size();
  for (size_t k = 0; k < m; ++k) {
    EF num = ef_one(), den = ef_one();
    for (size_t j = 0; j < m; ++j) {
      if (j == k) continue;
      num *= r - EF::from(j);
      den *= EF::from(k) - EF::from(j);
    }
    acc += evals[k] * num * ef_inv(den);
  }
  return acc;
}
inline bool sumcheck_verify(EF claim, const SumcheckProof& pf, Oracle& o,
                            std::vector<EF>* challenges) {
  EF cur = claim;
  challenges->clear();
  for (auto& ev : pf.round_polys) {
    if (ev.size() < 2 || ev[0] + ev[1] != cur) return false;
    EF r = o.next_field();
    cur = interpolate(ev, r);
    challenges->push_back(r);
  }
  EF prod = ef_one();
  for (auto& f : pf.final_evals) prod *= f;
  return prod == cur;
}

template <class T>
inline std::vector<T> rev(const std::vector<T>& v) {
  return std::vector<T>(v.rbegin(), v.rend());
}
template <class T>
inline std::vector<T> cat(const std::vector<T>& lo, const std::vector<T>& hi) {
  std::vector<T> o(lo);
  o.insert(o.end(), hi.begin(), hi.end());
  return o;
}

}  // namespace orc
