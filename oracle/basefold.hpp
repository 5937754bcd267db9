// ORACLE (test infrastructure only): the Basefold secondary PCS of pcs/src/basefold.rs —
// interleaved-RS commit (`to_commit`, `commit_{base,ext}_on_domain`, :257-382), the standalone
// open/verify (:384-642) and the shared-domain batched open/verify (:648-1035).
#pragma once
#include <algorithm>
#include <map>
#include <vector>

#include "merkle.hpp"
#include "poly.hpp"

namespace orc {

constexpr unsigned LOG_INTERLEAVE = 6;  // basefold.rs:15-16

inline size_t query_num(size_t code_rate) { return (100 + code_rate - 1) / code_rate; }  // :107

inline std::vector<uint8_t> ser_leaf(const std::vector<u64>& v) { return serialize_bf(v); }
inline std::vector<uint8_t> ser_leaf(const std::vector<EF>& v) { return serialize_ef(v); }
inline void dft_any(std::vector<u64>& a) { dft_bf(a); }
inline void dft_any(std::vector<EF>& a) { dft_ef(a); }
template <class T> inline T zero_of();
template <> inline u64 zero_of<u64>() { return 0; }
template <> inline EF zero_of<EF>() { return ef_zero(); }

template <class LF>
struct BasefoldState {
  std::vector<std::vector<LF>> codes;  // codes[j] = j-th interleaved codeword, length L
  MerkleTree tree;                     // leaf p = serialize(codes[0][p], ..., codes[2^li-1][p])
  std::vector<EF> poly;                // full polynomial (upcast to EF)
  unsigned num_vars = 0, code_rate = 0, log_interleave = 0;
};

// commit_{base,ext}_on_domain + to_commit (basefold.rs:257-307, 341-382).
template <class LF>
inline BasefoldState<LF> commit_on_domain(const std::vector<LF>& poly, unsigned code_rate,
                                          unsigned li, Hash* root) {
  BasefoldState<LF> st;
  auto chunks = mle_split(poly, poly.size() >> li);
  size_t code_len = chunks[0].size() << code_rate;
  parallel_ranges(chunks.size(), [&](size_t lo, size_t hi) {
    for (size_t j = lo; j < hi; ++j) {
      chunks[j].resize(code_len, zero_of<LF>());
      dft_any(chunks[j]);
    }
  });
  for (auto& c : chunks) st.codes.push_back(std::move(c));
  std::vector<Hash> lh(code_len);
  parallel_ranges(code_len, [&](size_t lo, size_t hi) {
    std::vector<LF> col(st.codes.size());
    for (size_t p = lo; p < hi; ++p) {
      for (size_t j = 0; j < st.codes.size(); ++j) col[j] = st.codes[j][p];
      auto bytes = ser_leaf(col);
      lh[p] = hash_bytes(bytes.data(), bytes.size());
    }
  }, size_t(1) << 10);
  st.tree = MerkleTree::from_leaf_hashes(std::move(lh));
  *root = st.tree.root();
  st.poly.reserve(poly.size());
  for (auto& x : poly) st.poly.push_back(lift(x));
  unsigned nv = 0;
  while ((size_t(1) << nv) < poly.size()) ++nv;
  st.num_vars = nv;
  st.code_rate = code_rate;
  st.log_interleave = li;
  return st;
}

// eq_fold_codeword (basefold.rs:201-218): out[i] = (1-r)(x+nx)/2 + r (x-nx) g^{-i} / 2.
inline std::vector<EF> eq_fold_codeword(const std::vector<EF>& v, EF r) {
  size_t len = v.size(), h = len / 2;
  unsigned lg = 0;
  while ((size_t(1) << lg) < len) ++lg;
  u64 g_inv = inv(two_adic_generator(lg));
  u64 inv2 = inv(2);
  u64 tw = 1;
  std::vector<EF> out;
  out.reserve(h);
  for (size_t i = 0; i < h; ++i) {
    EF x = v[i], nx = v[i + h];
    EF pe = (x + nx) * inv2;
    EF po = ((x - nx) * tw) * inv2;
    out.push_back((ef_one() - r) * pe + r * po);
    tw = mul(tw, g_inv);
  }
  return out;
}
inline EF eq_fold_at(EF a, EF b, EF r, size_t len, size_t pos) {  // basefold.rs:222-229
  unsigned lg = 0;
  while ((size_t(1) << lg) < len) ++lg;
  u64 tw = pow(inv(two_adic_generator(lg)), pos);
  u64 inv2 = inv(2);
  EF pe = (a + b) * inv2;
  EF po = ((a - b) * tw) * inv2;
  return (ef_one() - r) * pe + r * po;
}
inline std::vector<size_t> level_positions(const std::vector<size_t>& base, size_t half) {
  std::vector<size_t> pos;  // basefold.rs:234-244
  for (size_t idx : base) {
    pos.push_back(idx % half);
    pos.push_back(idx % half + half);
  }
  std::sort(pos.begin(), pos.end());
  pos.erase(std::unique(pos.begin(), pos.end()), pos.end());
  return pos;
}
inline std::vector<size_t> query_set(Oracle& o, size_t q, size_t modulus) {
  std::vector<size_t> base;
  for (u64 v : o.next_n_ints(q)) base.push_back((size_t)(v % modulus));
  std::sort(base.begin(), base.end());
  base.erase(std::unique(base.begin(), base.end()), base.end());
  return base;
}

template <class F>
struct Opening {  // RoundOpening / BaseOpening
  std::vector<uint8_t> proof_bytes;
  std::map<size_t, std::vector<F>> values;
};

template <class LF>
inline Opening<LF> open_base(const BasefoldState<LF>& st, const std::vector<size_t>& pos) {
  Opening<LF> op;
  op.proof_bytes = st.tree.open(pos);
  for (size_t p : pos) {
    std::vector<LF> col;
    for (auto& c : st.codes) col.push_back(c[p]);
    op.values[p] = col;
  }
  return op;
}
inline std::vector<MerkleTree> commit_levels(const std::vector<std::vector<EF>>& levels,
                                             size_t rounds, std::vector<Hash>* roots) {
  std::vector<MerkleTree> mts;
  for (size_t k = 1; k < rounds; ++k) {
    std::vector<Hash> lh;
    for (const EF& v : levels[k]) {
      auto b = serialize_ef({v});
      lh.push_back(hash_bytes(b.data(), b.size()));
    }
    mts.push_back(MerkleTree::from_leaf_hashes(std::move(lh)));
    roots->push_back(mts.back().root());
  }
  return mts;
}
inline std::vector<Opening<EF>> open_levels(const std::vector<MerkleTree>& mts,
                                            const std::vector<std::vector<EF>>& levels,
                                            const std::vector<size_t>& base, size_t l,
                                            size_t rounds) {
  std::vector<Opening<EF>> ops;
  for (size_t k = 1; k < rounds; ++k) {
    size_t cur_len = l >> k;
    auto positions = level_positions(base, cur_len / 2);
    Opening<EF> op;
    op.proof_bytes = mts[k - 1].open(positions);
    for (size_t p : positions) op.values[p] = {levels[k][p]};
    ops.push_back(std::move(op));
  }
  return ops;
}
template <class F>
inline bool verify_opening(const Opening<F>& op, const Hash& root, size_t leaves) {
  std::vector<size_t> idx;
  std::vector<std::vector<uint8_t>> lv;
  for (auto& kv : op.values) {
    idx.push_back(kv.first);
    lv.push_back(ser_leaf(kv.second));
  }
  if (idx.empty()) return false;
  return merkle_verify(root, op.proof_bytes, idx, lv, leaves);
}

// ---- standalone open (basefold.rs:84-103, 384-516) ----
template <class LF>
struct BasefoldProof {
  std::vector<std::pair<EF, EF>> reduction_msgs;
  std::vector<Hash> fold_roots;
  std::vector<EF> final_codeword;
  Opening<LF> base_opening;
  std::vector<Opening<EF>> fold_openings;
  EF claimed_eval;
  unsigned num_vars = 0, code_rate = 0, log_interleave = 0;
};

template <class LF>
inline BasefoldProof<LF> basefold_prove(const BasefoldState<LF>& st, const std::vector<EF>& pt,
                                        Oracle& o) {
  unsigned n = st.num_vars, li = st.log_interleave;
  if (pt.size() != n || n < li) throw std::runtime_error("basefold_prove: point size");
  size_t rounds = n - li, l = st.codes[0].size();
  BasefoldProof<LF> pf;
  pf.claimed_eval = mle_eval(st.poly, pt);
  auto eq4 = new_eq(std::vector<EF>(pt.begin(), pt.begin() + li));
  std::vector<EF> oracle0(l, ef_zero());
  for (size_t j = 0; j < st.codes.size(); ++j)
    for (size_t i = 0; i < l; ++i) oracle0[i] += eq4[j] * lift(st.codes[j][i]);
  std::vector<EF> m = st.poly;
  mle_fold(m, std::vector<EF>(pt.begin(), pt.begin() + li));
  std::vector<EF> zp(pt.begin() + li, pt.end());
  std::vector<std::vector<EF>> levels{oracle0};
  EF y = pf.claimed_eval;
  for (size_t round = 0; round < rounds; ++round) {
    size_t half = m.size() / 2;
    std::vector<EF> m0(half), m1(half);
    for (size_t i = 0; i < half; ++i) m0[i] = m[2 * i], m1[i] = m[2 * i + 1];
    std::vector<EF> rest(zp.begin() + round + 1, zp.end());
    EF l0 = mle_eval(m0, rest), l1 = mle_eval(m1, rest);
    if ((ef_one() - zp[round]) * l0 + zp[round] * l1 != y)
      throw std::runtime_error("basefold_prove: reduction check");  // debug_assert :432
    pf.reduction_msgs.push_back({l0, l1});
    EF r = o.next_field();
    y = (ef_one() - r) * l0 + r * l1;
    mle_fold(m, {r});
    levels.push_back(eq_fold_codeword(levels.back(), r));
  }
  pf.final_codeword = levels[rounds];
  auto mts = commit_levels(levels, rounds, &pf.fold_roots);
  auto base = query_set(o, query_num(st.code_rate), l / 2);
  pf.base_opening = open_base(st, level_positions(base, l / 2));
  pf.fold_openings = open_levels(mts, levels, base, l, rounds);
  pf.num_vars = n;
  pf.code_rate = st.code_rate;
  pf.log_interleave = li;
  return pf;
}

template <class LF>
inline bool basefold_verify(const Hash& commit, const std::vector<EF>& pt,
                            const BasefoldProof<LF>& pf, Oracle& o) {
  unsigned n = pf.num_vars, li = pf.log_interleave;
  if (pt.size() != n || n < li) return false;
  size_t rounds = n - li;
  size_t l = (size_t(1) << (n - li)) << pf.code_rate;
  if (pf.reduction_msgs.size() != rounds || pf.fold_roots.size() + 1 < rounds ||
      pf.fold_openings.size() + 1 < rounds || pf.final_codeword.empty())
    return false;
  auto eq4 = new_eq(std::vector<EF>(pt.begin(), pt.begin() + li));
  std::vector<EF> zp(pt.begin() + li, pt.end());
  EF y = pf.claimed_eval;
  std::vector<EF> ch;
  for (size_t round = 0; round < rounds; ++round) {
    EF l0 = pf.reduction_msgs[round].first, l1 = pf.reduction_msgs[round].second;
    if ((ef_one() - zp[round]) * l0 + zp[round] * l1 != y) return false;
    EF r = o.next_field();
    ch.push_back(r);
    y = (ef_one() - r) * l0 + r * l1;
  }
  auto base = query_set(o, query_num(pf.code_rate), l / 2);
  if (!verify_opening(pf.base_opening, commit, l)) return false;
  for (size_t k = 1; k < rounds; ++k)
    if (!verify_opening(pf.fold_openings[k - 1], pf.fold_roots[k - 1], l >> k)) return false;
  auto val_at = [&](size_t k, size_t p, bool* ok) -> EF {
    if (k == 0) {
      auto it = pf.base_opening.values.find(p);
      if (it == pf.base_opening.values.end() || it->second.size() != eq4.size()) {
        *ok = false;
        return ef_zero();
      }
      EF acc = ef_zero();
      for (size_t j = 0; j < it->second.size(); ++j) acc += eq4[j] * lift(it->second[j]);
      return acc;
    }
    auto it = pf.fold_openings[k - 1].values.find(p);
    if (it == pf.fold_openings[k - 1].values.end() || it->second.size() != 1) {
      *ok = false;
      return ef_zero();
    }
    return it->second[0];
  };
  size_t final_len = l >> rounds;
  if (pf.final_codeword.size() != final_len) return false;
  for (size_t idx : base) {
    bool have = false, ok = true;
    EF derived;
    for (size_t k = 0; k < rounds; ++k) {
      size_t cur = l >> k, half = cur / 2, pos = idx % half, sib = pos + half;
      EF a = val_at(k, pos, &ok), b = val_at(k, sib, &ok);
      if (!ok) return false;
      if (have) {
        size_t prev = idx % cur;
        if (derived != (prev == pos ? a : b)) return false;
      }
      derived = eq_fold_at(a, b, ch[k], cur, pos);
      have = true;
    }
    if (have && derived != pf.final_codeword[idx % final_len]) return false;
  }
  EF c0 = pf.final_codeword[0];
  for (auto& v : pf.final_codeword)
    if (v != c0) return false;
  return y == c0;
}

// ---- shared-domain batched open (basefold.rs:151-162, 648-856) ----
struct BatchProof {
  std::vector<std::vector<EF>> reduction_msgs;  // per channel, R entries (l0 only)
  std::vector<Hash> fold_roots;
  std::vector<EF> final_codeword;
  std::vector<Opening<EF>> fold_openings;
  std::vector<Opening<u64>> base_bf;
  std::vector<Opening<EF>> base_ef;
  unsigned code_rate = 0, log_len = 0;
};

struct Channel {
  std::vector<EF> oracle0, m, zp;
  EF y;
};
template <class LF>
inline Channel make_channel(const BasefoldState<LF>& st, const std::vector<EF>& pt, size_t d) {
  Channel c;  // basefold.rs:648-671
  unsigned li = st.log_interleave;
  auto eq4 = new_eq(std::vector<EF>(pt.begin(), pt.begin() + li));
  c.oracle0.assign(d, ef_zero());
  parallel_ranges(d, [&](size_t lo, size_t hi) {
    for (size_t j = 0; j < st.codes.size(); ++j)
      for (size_t i = lo; i < hi; ++i) c.oracle0[i] += eq4[j] * lift(st.codes[j][i]);
  }, size_t(1) << 12);
  c.m = st.poly;
  mle_fold(c.m, std::vector<EF>(pt.begin(), pt.begin() + li));
  c.y = mle_eval(st.poly, pt);
  c.zp.assign(pt.begin() + li, pt.end());
  return c;
}

inline BatchProof batch_prove(
    const std::vector<std::pair<const BasefoldState<u64>*, std::vector<EF>>>& bf,
    const std::vector<std::pair<const BasefoldState<EF>*, std::vector<EF>>>& ef, Oracle& o) {
  if (bf.empty() && ef.empty()) throw std::runtime_error("batch_prove needs a task");
  size_t d = bf.empty() ? ef[0].first->codes[0].size() : bf[0].first->codes[0].size();
  unsigned code_rate = bf.empty() ? ef[0].first->code_rate : bf[0].first->code_rate;
  for (auto& t : bf)
    if (t.first->codes[0].size() != d || t.first->code_rate != code_rate)
      throw std::runtime_error("batched commitments must share one RS domain");
  for (auto& t : ef)
    if (t.first->codes[0].size() != d || t.first->code_rate != code_rate)
      throw std::runtime_error("batched commitments must share one RS domain");
  unsigned log_len = 0;
  while ((size_t(1) << log_len) < d) ++log_len;
  size_t rounds = log_len - code_rate;
  std::vector<Channel> chs;
  for (auto& t : bf) {
    if (t.second.size() != t.first->num_vars) throw std::runtime_error("point size");
    chs.push_back(make_channel(*t.first, t.second, d));
  }
  for (auto& t : ef) {
    if (t.second.size() != t.first->num_vars) throw std::runtime_error("point size");
    chs.push_back(make_channel(*t.first, t.second, d));
  }
  for (auto& c : chs)
    if (c.zp.size() != rounds) throw std::runtime_error("batch: rounds mismatch");  // :715
  size_t nch = chs.size();
  auto coeffs = o.next_n_fields(nch);
  std::vector<EF> combined(d, ef_zero());
  for (size_t c = 0; c < nch; ++c)
    for (size_t i = 0; i < d; ++i) combined[i] += coeffs[c] * chs[c].oracle0[i];
  BatchProof pf;
  pf.reduction_msgs.assign(nch, {});
  std::vector<std::vector<EF>> levels{combined};
  for (size_t round = 0; round < rounds; ++round) {
    std::vector<std::pair<EF, EF>> l01;
    for (size_t c = 0; c < nch; ++c) {
      auto& m = chs[c].m;
      size_t half = m.size() / 2;
      std::vector<EF> m0(half), m1(half);
      for (size_t i = 0; i < half; ++i) m0[i] = m[2 * i], m1[i] = m[2 * i + 1];
      std::vector<EF> rest(chs[c].zp.begin() + round + 1, chs[c].zp.end());
      EF l0 = mle_eval(m0, rest), l1 = mle_eval(m1, rest);
      EF zi = chs[c].zp[round];
      if ((ef_one() - zi) * l0 + zi * l1 != chs[c].y)
        throw std::runtime_error("batch_prove: reduction check");  // debug_assert :757
      pf.reduction_msgs[c].push_back(l0);
      l01.push_back({l0, l1});
    }
    EF r = o.next_field();
    for (size_t c = 0; c < nch; ++c) {
      chs[c].y = (ef_one() - r) * l01[c].first + r * l01[c].second;
      mle_fold(chs[c].m, {r});
    }
    levels.push_back(eq_fold_codeword(levels.back(), r));
  }
  pf.final_codeword = levels[rounds];
  auto mts = commit_levels(levels, rounds, &pf.fold_roots);
  auto base = query_set(o, query_num(code_rate), d / 2);
  auto bpos = level_positions(base, d / 2);
  for (auto& t : bf) pf.base_bf.push_back(open_base(*t.first, bpos));
  for (auto& t : ef) pf.base_ef.push_back(open_base(*t.first, bpos));
  pf.fold_openings = open_levels(mts, levels, base, d, rounds);
  pf.code_rate = code_rate;
  pf.log_len = log_len;
  return pf;
}

struct BatchClaim {
  Hash commit;
  std::vector<EF> point;
  EF value;
  unsigned li;
};

inline bool batch_verify(const std::vector<BatchClaim>& bfc, const std::vector<BatchClaim>& efc,
                         const BatchProof& pf, Oracle& o) {  // basefold.rs:860-1035
  if (pf.log_len < pf.code_rate || pf.log_len > 40) return false;
  size_t d = size_t(1) << pf.log_len;
  size_t rounds = pf.log_len - pf.code_rate;
  size_t nbf = bfc.size(), nch = nbf + efc.size();
  size_t nlev = rounds ? rounds - 1 : 0;
  if (pf.reduction_msgs.size() != nch || pf.base_bf.size() != nbf ||
      pf.base_ef.size() != efc.size() || pf.fold_roots.size() != nlev ||
      pf.fold_openings.size() != nlev)
    return false;
  std::vector<std::vector<EF>> eq4s;
  std::vector<const BatchClaim*> cl;
  std::vector<EF> ys;
  for (auto& c : bfc) cl.push_back(&c);
  for (auto& c : efc) cl.push_back(&c);
  for (size_t c = 0; c < nch; ++c) {
    const BatchClaim& b = *cl[c];
    if (b.point.size() < b.li || b.point.size() - b.li != rounds ||
        pf.reduction_msgs[c].size() != rounds)
      return false;
    eq4s.push_back(new_eq(std::vector<EF>(b.point.begin(), b.point.begin() + b.li)));
    ys.push_back(b.value);
  }
  auto coeffs = o.next_n_fields(nch);
  std::vector<EF> ch;
  for (size_t round = 0; round < rounds; ++round) {
    EF r = o.next_field();
    ch.push_back(r);
    for (size_t c = 0; c < nch; ++c) {
      EF l0 = pf.reduction_msgs[c][round];
      EF zi = cl[c]->point[cl[c]->li + round];
      if (zi == ef_zero()) return false;
      EF l1 = (ys[c] - (ef_one() - zi) * l0) * ef_inv(zi);
      ys[c] = (ef_one() - r) * l0 + r * l1;
    }
  }
  auto base = query_set(o, query_num(pf.code_rate), d / 2);
  auto bpos = level_positions(base, d / 2);
  auto keys_of = [](const auto& op) {
    std::vector<size_t> k;
    for (auto& kv : op.values) k.push_back(kv.first);
    return k;
  };
  for (size_t i = 0; i < nbf; ++i) {
    if (keys_of(pf.base_bf[i]) != bpos) return false;
    if (!verify_opening(pf.base_bf[i], bfc[i].commit, d)) return false;
  }
  for (size_t i = 0; i < efc.size(); ++i) {
    if (keys_of(pf.base_ef[i]) != bpos) return false;
    if (!verify_opening(pf.base_ef[i], efc[i].commit, d)) return false;
  }
  for (size_t k = 1; k < rounds; ++k)
    if (!verify_opening(pf.fold_openings[k - 1], pf.fold_roots[k - 1], d >> k)) return false;
  bool ok = true;
  auto val_at = [&](size_t k, size_t p) -> EF {
    if (k == 0) {
      EF acc = ef_zero();
      for (size_t c = 0; c < nch; ++c) {
        EF a = ef_zero();
        if (c < nbf) {
          auto it = pf.base_bf[c].values.find(p);
          if (it == pf.base_bf[c].values.end() || it->second.size() != eq4s[c].size()) {
            ok = false;
            return ef_zero();
          }
          for (size_t j = 0; j < it->second.size(); ++j) a += eq4s[c][j] * lift(it->second[j]);
        } else {
          auto it = pf.base_ef[c - nbf].values.find(p);
          if (it == pf.base_ef[c - nbf].values.end() || it->second.size() != eq4s[c].size()) {
            ok = false;
            return ef_zero();
          }
          for (size_t j = 0; j < it->second.size(); ++j) a += eq4s[c][j] * it->second[j];
        }
        acc += coeffs[c] * a;
      }
      return acc;
    }
    auto it = pf.fold_openings[k - 1].values.find(p);
    if (it == pf.fold_openings[k - 1].values.end() || it->second.size() != 1) {
      ok = false;
      return ef_zero();
    }
    return it->second[0];
  };
  size_t final_len = d >> rounds;
  if (pf.final_codeword.size() != final_len) return false;
  for (size_t idx : base) {
    bool have = false;
    EF derived;
    for (size_t k = 0; k < rounds; ++k) {
      size_t cur = d >> k, half = cur / 2, pos = idx % half, sib = pos + half;
      EF a = val_at(k, pos), b = val_at(k, sib);
      if (!ok) return false;
      if (have && derived != ((idx % cur) == pos ? a : b)) return false;
      derived = eq_fold_at(a, b, ch[k], cur, pos);
      have = true;
    }
    if (have && derived != pf.final_codeword[idx % final_len]) return false;
  }
  EF c0 = pf.final_codeword[0];
  for (auto& v : pf.final_codeword)
    if (v != c0) return false;
  EF comb = ef_zero();
  for (size_t c = 0; c < nch; ++c) comb += coeffs[c] * ys[c];
  return comb == c0;
}

}  // namespace orc
