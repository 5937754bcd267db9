// ORACLE (test infrastructure only): a single-threaded CPU restatement of the GKR fraction-sum
// circuit and the GKR-LogUp lookup built on it (logup/src/frac_sum.rs, logup/src/lookup.rs).
// Only tests/, the smoke check and bench.py's CPU-baseline leg load this code, and only as the
// checker; the product library never links it.
//
// The reference keeps these proofs as Rust structs; the byte layout below is the boundary's own,
// written identically by the product library:
//   FracSumProof  "LGSF" u32:version=1, num:EF, den:EF, u32 nlayers,
//                 per layer: u32 rounds, rounds x 4 EF (g(0), g(1), g(2), g(3)), 4 EF leaves
//                 (A0, A1, B0, B1)
//   LookupProof   "LGSL" u32:version=1, query:FracSumProof, table:FracSumProof
#pragma once
#include <array>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "proof_io.hpp"

namespace orc {

struct FsLayer {
  std::vector<std::array<EF, 4>> round_polys;
  std::array<EF, 4> leaves;
};
struct FracSumProof {
  EF num, den;
  std::vector<FsLayer> layers;
};
struct FsClaim {  // the reduced input claim (point low-bit-first, p_in(point), q_in(point))
  std::vector<EF> point;
  EF p, q;
};

// eq_table (frac_sum.rs:56-69): z[0] is the low bit, each later coordinate a new high bit.
inline std::vector<EF> fs_eq_table(const std::vector<EF>& z) {
  std::vector<EF> tab{ef_one()};
  for (const EF& zk : z) {
    const size_t half = tab.size();
    std::vector<EF> next(half * 2);
    for (size_t i = 0; i < half; ++i) {
      next[i] = tab[i] * (ef_one() - zk);
      next[i + half] = tab[i] * zk;
    }
    tab.swap(next);
  }
  return tab;
}
// eq_eval (frac_sum.rs:72-76)
inline EF fs_eq_eval(const std::vector<EF>& z, const std::vector<EF>& zp) {
  EF acc = ef_one();
  for (size_t i = 0; i < z.size() && i < zp.size(); ++i)
    acc = acc * (z[i] * zp[i] + (ef_one() - z[i]) * (ef_one() - zp[i]));
  return acc;
}
// fold_low (frac_sum.rs:79-85)
inline void fs_fold_low(std::vector<EF>& a, const EF& c) {
  const size_t half = a.size() / 2;
  for (size_t j = 0; j < half; ++j) a[j] = a[2 * j] + c * (a[2 * j + 1] - a[2 * j]);
  a.resize(half);
}
// interp4 (frac_sum.rs:88-106): the degree-3 polynomial through (0..3, ev) at x, Lagrange form
// with denominators -6, 2, -2, 6.
inline EF fs_interp4(const std::array<EF, 4>& ev, const EF& x) {
  const EF two = ef_one() + ef_one(), three = two + ef_one(), six = two * three;
  const EF nodes[4] = {ef_zero(), ef_one(), two, three};
  const EF denoms[4] = {ef_zero() - six, two, ef_zero() - two, six};
  EF acc = ef_zero();
  for (int k = 0; k < 4; ++k) {
    EF num = ef_one();
    for (int m = 0; m < 4; ++m)
      if (m != k) num = num * (x - nodes[m]);
    acc = acc + ev[k] * num * ef_inv(denoms[k]);
  }
  return acc;
}

// prove_layer (frac_sum.rs:165-218)
inline FsLayer fs_prove_layer(const std::vector<EF>& z, const EF& lambda,
                              const std::vector<EF>& pn, const std::vector<EF>& qn, Oracle& o,
                              std::vector<EF>* zprime) {
  const size_t r = z.size(), half0 = pn.size() / 2;
  std::vector<EF> a0(half0), a1(half0), b0(half0), b1(half0);
  for (size_t i = 0; i < half0; ++i) {
    a0[i] = pn[2 * i];
    a1[i] = pn[2 * i + 1];
    b0[i] = qn[2 * i];
    b1[i] = qn[2 * i + 1];
  }
  std::vector<EF> eqv = fs_eq_table(z);
  const EF two = ef_one() + ef_one(), three = two + ef_one();
  const EF pts[4] = {ef_zero(), ef_one(), two, three};
  FsLayer L;
  zprime->clear();
  for (size_t round = 0; round < r; ++round) {
    const size_t half = eqv.size() / 2;
    std::array<EF, 4> g{};
    for (size_t j = 0; j < half; ++j) {
      for (int t = 0; t < 4; ++t) {
        const EF& p = pts[t];
        EF e = eqv[2 * j] + p * (eqv[2 * j + 1] - eqv[2 * j]);
        EF av0 = a0[2 * j] + p * (a0[2 * j + 1] - a0[2 * j]);
        EF av1 = a1[2 * j] + p * (a1[2 * j + 1] - a1[2 * j]);
        EF bv0 = b0[2 * j] + p * (b0[2 * j + 1] - b0[2 * j]);
        EF bv1 = b1[2 * j] + p * (b1[2 * j + 1] - b1[2 * j]);
        g[t] = g[t] + e * (av0 * bv1 + av1 * bv0 + lambda * bv0 * bv1);
      }
    }
    L.round_polys.push_back(g);
    const EF c = o.next_field();
    zprime->push_back(c);
    fs_fold_low(a0, c);
    fs_fold_low(a1, c);
    fs_fold_low(b0, c);
    fs_fold_low(b1, c);
    fs_fold_low(eqv, c);
  }
  L.leaves = {a0[0], a1[0], b0[0], b1[0]};
  return L;
}

// prove (frac_sum.rs:110-161)
inline FracSumProof frac_sum_prove(const std::vector<EF>& p_in, const std::vector<EF>& q_in,
                                   Oracle& o, FsClaim* claim) {
  const size_t n = p_in.size();
  if (n == 0 || (n & (n - 1)) || q_in.size() != n)
    throw std::runtime_error("frac_sum: inputs of one power-of-two length");
  unsigned k = 0;
  while ((size_t(1) << k) < n) ++k;
  std::vector<std::vector<EF>> lp(k + 1), lq(k + 1);
  lp[k] = p_in;
  lq[k] = q_in;
  for (int s = (int)k - 1; s >= 0; --s) {
    const size_t sz = size_t(1) << s;
    lp[s].resize(sz);
    lq[s].resize(sz);
    for (size_t i = 0; i < sz; ++i) {
      const auto &pn = lp[s + 1], &qn = lq[s + 1];
      lp[s][i] = pn[2 * i] * qn[2 * i + 1] + pn[2 * i + 1] * qn[2 * i];
      lq[s][i] = qn[2 * i] * qn[2 * i + 1];
    }
  }
  FracSumProof pf;
  pf.num = lp[0][0];
  pf.den = lq[0][0];
  std::vector<EF> z, zp;
  for (unsigned r = 0; r < k; ++r) {
    const EF lambda = o.next_field();
    FsLayer L = fs_prove_layer(z, lambda, lp[r + 1], lq[r + 1], o, &zp);
    const EF beta = o.next_field();
    z.clear();
    z.push_back(beta);
    z.insert(z.end(), zp.begin(), zp.end());
    pf.layers.push_back(L);
    if (r + 1 == k) {
      claim->point = z;
      claim->p = (ef_one() - beta) * L.leaves[0] + beta * L.leaves[1];
      claim->q = (ef_one() - beta) * L.leaves[2] + beta * L.leaves[3];
      return pf;
    }
  }
  claim->point.clear();  // k == 0: the root itself at the empty point
  claim->p = pf.num;
  claim->q = pf.den;
  return pf;
}

// verify (frac_sum.rs:221-258); false where the reference returns None.
inline bool frac_sum_verify(const FracSumProof& pf, Oracle& o, FsClaim* claim) {
  const size_t k = pf.layers.size();
  std::vector<EF> z;
  EF p_cur = pf.num, q_cur = pf.den;
  for (size_t r = 0; r < k; ++r) {
    const EF lambda = o.next_field();
    const FsLayer& L = pf.layers[r];
    if (L.round_polys.size() != r) return false;
    EF cur = p_cur + lambda * q_cur;
    std::vector<EF> zp;
    for (const auto& poly : L.round_polys) {
      if (poly[0] + poly[1] != cur) return false;
      const EF c = o.next_field();
      cur = fs_interp4(poly, c);
      zp.push_back(c);
    }
    const EF a0 = L.leaves[0], a1 = L.leaves[1], b0 = L.leaves[2], b1 = L.leaves[3];
    if (cur != fs_eq_eval(z, zp) * (a0 * b1 + a1 * b0 + lambda * b0 * b1)) return false;
    const EF beta = o.next_field();
    z.clear();
    z.push_back(beta);
    z.insert(z.end(), zp.begin(), zp.end());
    p_cur = (ef_one() - beta) * a0 + beta * a1;
    q_cur = (ef_one() - beta) * b0 + beta * b1;
  }
  claim->point = z;
  claim->p = p_cur;
  claim->q = q_cur;
  return true;
}

// ---- GKR-LogUp lookup (logup/src/lookup.rs) --------------------------------------------------
struct LookupProof {
  FracSumProof query, table;
};
struct LookupClaims {  // OpeningClaims of lookup.rs:221-228: a(zq), e(zt), t(zt)
  std::vector<EF> zq, zt;
  EF a, e, t;
};

// prove_with_opening_points (lookup.rs:119-143)
inline LookupProof lookup_prove(const std::vector<EF>& a, const std::vector<EF>& t,
                                const std::vector<EF>& e, Oracle& o, std::vector<EF>* zq,
                                std::vector<EF>* zt) {
  if ((a.size() & (a.size() - 1)) || (t.size() & (t.size() - 1)) || a.empty() || t.empty())
    throw std::runtime_error("lookup: power-of-two lengths");
  if (e.size() != t.size()) throw std::runtime_error("lookup: |e| != |t|");
  const EF alpha = o.next_field();
  std::vector<EF> pq(a.size(), ef_one()), qq(a.size()), qt(t.size());
  for (size_t i = 0; i < a.size(); ++i) qq[i] = alpha - a[i];
  FsClaim cq, ct;
  LookupProof pf;
  pf.query = frac_sum_prove(pq, qq, o, &cq);
  for (size_t j = 0; j < t.size(); ++j) qt[j] = alpha - t[j];
  pf.table = frac_sum_prove(e, qt, o, &ct);
  *zq = cq.point;
  *zt = ct.point;
  return pf;
}

// verify (lookup.rs:191-229)
inline bool lookup_verify(const LookupProof& pf, Oracle& o, LookupClaims* out) {
  const EF alpha = o.next_field();
  FsClaim cq, ct;
  if (!frac_sum_verify(pf.query, o, &cq)) return false;
  if (!frac_sum_verify(pf.table, o, &ct)) return false;
  if (cq.p != ef_one()) return false;
  if (pf.query.num * pf.table.den != pf.table.num * pf.query.den) return false;
  out->zq = cq.point;
  out->zt = ct.point;
  out->a = alpha - cq.q;
  out->e = ct.p;
  out->t = alpha - ct.q;
  return true;
}

// multiplicities (lookup.rs:66-76): count of each table entry among the queries, first match.
inline std::vector<EF> lookup_multiplicities(const std::vector<EF>& a, const std::vector<EF>& t) {
  std::vector<u64> cnt(t.size(), 0);
  for (const EF& ai : a)
    for (size_t j = 0; j < t.size(); ++j)
      if (t[j] == ai) {
        ++cnt[j];
        break;
      }
  std::vector<EF> e(t.size());
  for (size_t j = 0; j < t.size(); ++j) e[j] = EF::from(cnt[j] % P);
  return e;
}

// ---- byte layout ---------------------------------------------------------------------------
inline void encode_frac_sum(Writer& w, const FracSumProof& pf) {
  w.u32(0x4653474C);  // "LGSF"
  w.u32(1);
  w.ef(pf.num);
  w.ef(pf.den);
  w.u32((uint32_t)pf.layers.size());
  for (const FsLayer& L : pf.layers) {
    w.u32((uint32_t)L.round_polys.size());
    for (const auto& g : L.round_polys)
      for (const EF& v : g) w.ef(v);
    for (const EF& v : L.leaves) w.ef(v);
  }
}
inline bool decode_frac_sum(Reader& r, FracSumProof* pf) {
  if (r.u32() != 0x4653474C || r.u32() != 1) return false;
  pf->num = r.ef();
  pf->den = r.ef();
  const uint32_t nl = r.u32();
  if (!r.ok || nl > 64) return false;
  pf->layers.assign(nl, FsLayer{});
  for (uint32_t l = 0; l < nl && r.ok; ++l) {
    const uint32_t nr = r.u32();
    if (!r.ok || nr > 64) return false;
    pf->layers[l].round_polys.resize(nr);
    for (auto& g : pf->layers[l].round_polys)
      for (EF& v : g) v = r.ef();
    for (EF& v : pf->layers[l].leaves) v = r.ef();
  }
  return r.ok;
}
inline std::vector<uint8_t> encode_frac_sum_proof(const FracSumProof& pf) {
  Writer w;
  encode_frac_sum(w, pf);
  return w.b;
}
inline std::vector<uint8_t> encode_lookup_proof(const LookupProof& pf) {
  Writer w;
  w.u32(0x4C53474C);  // "LGSL"
  w.u32(1);
  encode_frac_sum(w, pf.query);
  encode_frac_sum(w, pf.table);
  return w.b;
}
inline bool decode_lookup_proof(const uint8_t* p, size_t n, LookupProof* pf) {
  Reader r(p, n);
  if (r.u32() != 0x4C53474C || r.u32() != 1) return false;
  if (!decode_frac_sum(r, &pf->query) || !decode_frac_sum(r, &pf->table)) return false;
  return r.ok && r.pos == n;
}
inline bool decode_frac_sum_proof(const uint8_t* p, size_t n, FracSumProof* pf) {
  Reader r(p, n);
  return decode_frac_sum(r, pf) && r.pos == n;
}

}  // namespace orc
