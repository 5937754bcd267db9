// Host verifier of the prover library: Ligesis::verify (pcs/src/ligesis.rs:569-756) with
// sumcheck::verify (utils/src/sumcheck.rs:88-130), Basefold::batch_verify
// (pcs/src/basefold.rs:860-1035) and Merkle multiproof checks (utils/src/merkle.rs:89-103).
// The verifier is cheap CPU work in the reference as well; it runs on the caller's thread.
#include <map>
#include <stdexcept>

#include "blake3.cuh"
#include "proof.hpp"

namespace lgs {

namespace {

using EFv = std::vector<ef2>;

ef2 E(u64 a) { return ef_make(a, 0); }
ef2 lift_value(u64 a) { return ef_make(a, 0); }
ef2 lift_value(const ef2& a) { return a; }

EFv new_eq(const EFv& p) {
  EFv ev{ef_one()};
  for (size_t t = p.size(); t-- > 0;) {
    EFv nx;
    nx.reserve(ev.size() * 2);
    for (const ef2& x : ev) {
      nx.push_back(ef_mul(ef_sub(ef_one(), p[t]), x));
      nx.push_back(ef_mul(p[t], x));
    }
    ev.swap(nx);
  }
  return ev;
}
ef2 eval_eq(const EFv& a, const EFv& b) {
  ef2 r = ef_one();
  for (size_t i = 0; i < std::min(a.size(), b.size()); ++i)
    r = ef_mul(r, ef_add(ef_mul(a[i], b[i]), ef_mul(ef_sub(ef_one(), a[i]), ef_sub(ef_one(), b[i]))));
  return r;
}
ef2 mle_eval(EFv s, const EFv& pt) {
  if (((size_t)1 << pt.size()) != s.size()) throw std::runtime_error("mle size");
  size_t cur = s.size() >> 1;
  for (const ef2& r : pt) {
    for (size_t i = 0; i < cur; ++i) s[i] = ef_lerp(s[2 * i], s[2 * i + 1], r);
    cur >>= 1;
  }
  return s[0];
}
EFv rev(EFv v) {
  std::reverse(v.begin(), v.end());
  return v;
}
EFv cat(EFv a, const EFv& b) {
  a.insert(a.end(), b.begin(), b.end());
  return a;
}

struct Oracle {
  const u64* f;
  size_t nf, fi;
  const uint64_t* ints;
  size_t ni, ii;
  ef2 field() {
    if (fi >= nf) throw std::runtime_error("oracle exhausted");
    ef2 e = ef_make(f[2 * fi], f[2 * fi + 1]);
    ++fi;
    return e;
  }
  EFv fields(size_t k) {
    EFv v;
    for (size_t i = 0; i < k; ++i) v.push_back(field());
    return v;
  }
  const uint64_t* take_ints(size_t k) {
    if (ii + k > ni) throw std::runtime_error("oracle exhausted");
    const uint64_t* p = ints + ii;
    ii += k;
    return p;
  }
};

ef2 interpolate(const EFv& ev, ef2 r) {
  ef2 acc = ef_zero();
  for (size_t k = 0; k < ev.size(); ++k) {
    ef2 num = ef_one(), den = ef_one();
    for (size_t j = 0; j < ev.size(); ++j) {
      if (j == k) continue;
      num = ef_mul(num, ef_sub(r, E(j)));
      den = ef_mul(den, ef_sub(E(k), E(j)));
    }
    acc = ef_add(acc, ef_mul(ef_mul(ev[k], num), ef_inv(den)));
  }
  return acc;
}
bool sc_verify(ef2 claim, const ScProof& p, Oracle& o, EFv* ch) {
  ef2 cur = claim;
  ch->clear();
  for (auto& ev : p.rounds) {
    if (ev.size() < 2 || !ef_eq(ef_add(ev[0], ev[1]), cur)) return false;
    ef2 r = o.field();
    cur = interpolate(ev, r);
    ch->push_back(r);
  }
  ef2 prod = ef_one();
  for (auto& f : p.finals) prod = ef_mul(prod, f);
  return ef_eq(prod, cur);
}

Hash32 hash_bytes(const std::vector<uint8_t>& b) {
  u32 out[8];
  auto word = [&](u32 i) {
    return (u32)b[4 * i] | ((u32)b[4 * i + 1] << 8) | ((u32)b[4 * i + 2] << 16) |
           ((u32)b[4 * i + 3] << 24);
  };
  b3_hash_words(word, (u32)b.size(), out);
  Hash32 h;
  std::memcpy(h.b, out, 32);
  return h;
}
Hash32 hash_pair(const Hash32& l, const Hash32& r) {
  u32 lw[8], rw[8], o[8];
  std::memcpy(lw, l.b, 32);
  std::memcpy(rw, r.b, 32);
  b3_parent(lw, rw, o);
  Hash32 h;
  std::memcpy(h.b, o, 32);
  return h;
}
void ser(std::vector<uint8_t>& b, u64 v) {
  for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i)));
}
std::vector<uint8_t> leaf_bytes(const std::vector<u64>& v) {
  std::vector<uint8_t> b;
  for (u64 x : v) ser(b, x);
  return b;
}
std::vector<uint8_t> leaf_bytes(const std::vector<ef2>& v) {
  std::vector<uint8_t> b;
  for (auto& x : v) ser(b, x.c0), ser(b, x.c1);
  return b;
}

// rs_merkle root reconstruction from sorted distinct indices (power-of-two trees).
bool merkle_check(const Hash32& root, const std::vector<uint8_t>& proof,
                  const std::vector<uint64_t>& idx, const std::vector<Hash32>& leaves,
                  uint64_t nleaves) {
  if (idx.empty() || idx.size() != leaves.size() || proof.size() % 32) return false;
  if (nleaves == 0 || (nleaves & (nleaves - 1))) return false;
  for (size_t i = 0; i < idx.size(); ++i)
    if (idx[i] >= nleaves || (i && idx[i] <= idx[i - 1])) return false;
  std::map<uint64_t, Hash32> known;
  for (size_t i = 0; i < idx.size(); ++i) known[idx[i]] = leaves[i];
  size_t pos = 0;
  for (uint64_t len = nleaves; len > 1; len >>= 1) {
    std::vector<uint64_t> cur;
    for (auto& kv : known) cur.push_back(kv.first);
    for (uint64_t i : cur) {
      uint64_t s = i ^ 1;
      if (!known.count(s)) {
        if (pos + 32 > proof.size()) return false;
        Hash32 h;
        std::memcpy(h.b, proof.data() + pos, 32);
        pos += 32;
        known[s] = h;
      }
    }
    std::map<uint64_t, Hash32> next;
    for (auto& kv : known)
      if (!(kv.first & 1)) next[kv.first / 2] = hash_pair(kv.second, known[kv.first + 1]);
    known.swap(next);
  }
  return pos == proof.size() && known.size() == 1 && known.begin()->second == root;
}
template <class F>
bool opening_check(const OpeningH<F>& op, const Hash32& root, uint64_t nleaves) {
  std::vector<uint64_t> idx;
  std::vector<Hash32> lh;
  for (auto& kv : op.values) {
    idx.push_back(kv.first);
    lh.push_back(hash_bytes(leaf_bytes(kv.second)));
  }
  return merkle_check(root, op.proof, idx, lh, nleaves);
}

ef2 eq_fold_at(ef2 a, ef2 b, ef2 r, uint64_t len, uint64_t pos) {
  u64 g = gl_two_adic_generator(ilog2_u64(len));
  u64 tw = gl_pow(gl_inv(g), pos);
  u64 inv2 = gl_inv(2);
  ef2 pe = ef_scale(ef_add(a, b), inv2);
  ef2 po = ef_scale(ef_scale(ef_sub(a, b), tw), inv2);
  return ef_add(ef_mul(ef_sub(ef_one(), r), pe), ef_mul(r, po));
}

struct Claim {
  Hash32 com;
  EFv point;
  ef2 value;
  unsigned li;
};

bool batch_verify(const std::vector<Claim>& bfc, const std::vector<Claim>& efc,
                  const BatchProofH& pf, Oracle& o) {
  if (pf.log_len < pf.code_rate || pf.log_len > 40) return false;
  const uint64_t d = (uint64_t)1 << pf.log_len;
  const size_t rounds = pf.log_len - pf.code_rate, nlev = rounds ? rounds - 1 : 0;
  const size_t nbf = bfc.size(), nch = nbf + efc.size();
  if (pf.msgs.size() != nch || pf.base_bf.size() != nbf || pf.base_ef.size() != efc.size() ||
      pf.fold_roots.size() != nlev || pf.fold_openings.size() != nlev)
    return false;
  std::vector<const Claim*> cl;
  for (auto& c : bfc) cl.push_back(&c);
  for (auto& c : efc) cl.push_back(&c);
  std::vector<EFv> eq4;
  EFv ys;
  for (size_t c = 0; c < nch; ++c) {
    if (cl[c]->point.size() < cl[c]->li || cl[c]->point.size() - cl[c]->li != rounds ||
        pf.msgs[c].size() != rounds)
      return false;
    eq4.push_back(new_eq(EFv(cl[c]->point.begin(), cl[c]->point.begin() + cl[c]->li)));
    ys.push_back(cl[c]->value);
  }
  EFv coeffs = o.fields(nch);
  EFv ch;
  for (size_t t = 0; t < rounds; ++t) {
    ef2 r = o.field();
    ch.push_back(r);
    for (size_t c = 0; c < nch; ++c) {
      ef2 l0 = pf.msgs[c][t], zi = cl[c]->point[cl[c]->li + t];
      if (ef_eq(zi, ef_zero())) return false;
      ef2 l1 = ef_mul(ef_sub(ys[c], ef_mul(ef_sub(ef_one(), zi), l0)), ef_inv(zi));
      ys[c] = ef_add(ef_mul(ef_sub(ef_one(), r), l0), ef_mul(r, l1));
    }
  }
  auto base = query_base(o.take_ints(QUERIES), d / 2);
  auto bpos = level_positions(base, d / 2);
  auto keys = [](const auto& op) {
    std::vector<uint64_t> k;
    for (auto& kv : op.values) k.push_back(kv.first);
    return k;
  };
  for (size_t i = 0; i < nbf; ++i)
    if (keys(pf.base_bf[i]) != bpos || !opening_check(pf.base_bf[i], bfc[i].com, d)) return false;
  for (size_t i = 0; i < efc.size(); ++i)
    if (keys(pf.base_ef[i]) != bpos || !opening_check(pf.base_ef[i], efc[i].com, d)) return false;
  for (size_t k = 1; k < rounds; ++k)
    if (!opening_check(pf.fold_openings[k - 1], pf.fold_roots[k - 1], d >> k)) return false;
  bool ok = true;
  auto find = [&](const auto& op, uint64_t p) -> decltype(&op.values[0].second) {
    auto it = std::lower_bound(op.values.begin(), op.values.end(), p,
                               [](const auto& kv, uint64_t x) { return kv.first < x; });
    if (it == op.values.end() || it->first != p) return nullptr;
    return &it->second;
  };
  auto val_at = [&](size_t k, uint64_t p) -> ef2 {
    if (k == 0) {
      ef2 acc = ef_zero();
      for (size_t c = 0; c < nch; ++c) {
        ef2 a = ef_zero();
        if (c < nbf) {
          auto v = find(pf.base_bf[c], p);
          if (!v || v->size() != eq4[c].size()) return ok = false, ef_zero();
          for (size_t j = 0; j < v->size(); ++j) a = ef_add(a, ef_scale(eq4[c][j], (*v)[j]));
        } else {
          auto v = find(pf.base_ef[c - nbf], p);
          if (!v || v->size() != eq4[c].size()) return ok = false, ef_zero();
          for (size_t j = 0; j < v->size(); ++j) a = ef_add(a, ef_mul(eq4[c][j], (*v)[j]));
        }
        acc = ef_add(acc, ef_mul(coeffs[c], a));
      }
      return acc;
    }
    auto v = find(pf.fold_openings[k - 1], p);
    if (!v || v->size() != 1) return ok = false, ef_zero();
    return (*v)[0];
  };
  const uint64_t final_len = d >> rounds;
  if (pf.final_codeword.size() != final_len) return false;
  for (uint64_t idx : base) {
    bool have = false;
    ef2 der = ef_zero();
    for (size_t k = 0; k < rounds; ++k) {
      uint64_t cur = d >> k, half = cur / 2, pos = idx % half;
      ef2 a = val_at(k, pos), b = val_at(k, pos + half);
      if (!ok) return false;
      if (have && !ef_eq(der, (idx % cur) == pos ? a : b)) return false;
      der = eq_fold_at(a, b, ch[k], cur, pos);
      have = true;
    }
    if (have && !ef_eq(der, pf.final_codeword[idx % final_len])) return false;
  }
  for (auto& v : pf.final_codeword)
    if (!ef_eq(v, pf.final_codeword[0])) return false;
  ef2 comb = ef_zero();
  for (size_t c = 0; c < nch; ++c) comb = ef_add(comb, ef_mul(coeffs[c], ys[c]));
  return ef_eq(comb, pf.final_codeword[0]);
}

// The level-0 value at leaf p of a standalone Basefold proof: sum_j eq4[j] leaf[j].
template <class F>
bool base_value(const OpeningH<F>& op, uint64_t p, const EFv& eq4, ef2* out) {
  auto it = std::lower_bound(op.values.begin(), op.values.end(), p,
                             [](const std::pair<uint64_t, std::vector<F>>& kv, uint64_t k) {
                               return kv.first < k;
                             });
  if (it == op.values.end() || it->first != p || it->second.size() != eq4.size()) return false;
  ef2 acc = ef_zero();
  for (size_t j = 0; j < eq4.size(); ++j) acc = ef_add(acc, ef_mul(eq4[j], lift_value(it->second[j])));
  *out = acc;
  return true;
}

}  // namespace

// Basefold::verify (pcs/src/basefold.rs:518-642): 1 accept, 0 reject.
int basefold_verify_host(const Hash32& root, const u64* point, size_t plen, const uint8_t* proof,
                         size_t proof_len, const u64* fields, size_t nfields,
                         const uint64_t* ints, size_t nints, uint64_t cursors[2]) {
  BasefoldProofH pf;
  if (!decode_basefold_proof(proof, proof_len, &pf)) return 0;
  const unsigned n = pf.num_vars, li = pf.log_interleave;
  if (plen != n || n <= li || n - li + pf.code_rate > 40) return 0;
  const unsigned rounds = n - li;
  const uint64_t l = ((uint64_t)1 << (n - li)) << pf.code_rate;
  if (pf.msgs.size() != rounds || pf.roots.size() + 1 != rounds || pf.folds.size() + 1 != rounds ||
      pf.final_codeword.size() != (l >> rounds))
    return 0;
  Oracle o{fields, nfields, (size_t)cursors[0], ints, nints, (size_t)cursors[1]};
  EFv pt(n);
  for (unsigned i = 0; i < n; ++i) pt[i] = ef_make(gl_canon(point[2 * i]), gl_canon(point[2 * i + 1]));
  auto run = [&]() -> bool {
    const EFv eq4 = new_eq(EFv(pt.begin(), pt.begin() + li));
    // evaluation-reduction claim chain
    ef2 y = pf.claimed;
    EFv ch;
    for (unsigned t = 0; t < rounds; ++t) {
      const ef2 l0 = pf.msgs[t].first, l1 = pf.msgs[t].second, zi = pt[li + t];
      if (!ef_eq(ef_add(ef_mul(ef_sub(ef_one(), zi), l0), ef_mul(zi, l1)), y)) return false;
      const ef2 r = o.field();
      ch.push_back(r);
      y = ef_add(ef_mul(ef_sub(ef_one(), r), l0), ef_mul(r, l1));
    }
    const size_t q = (100 + pf.code_rate - 1) / pf.code_rate;
    const uint64_t* qi = o.take_ints(q);
    std::vector<uint64_t> base;
    for (size_t t = 0; t < q; ++t) base.push_back(qi[t] % (l / 2));
    std::sort(base.begin(), base.end());
    base.erase(std::unique(base.begin(), base.end()), base.end());
    // Merkle openings: level 0 in the leaf field, folded levels in EF
    if (pf.leaf_ef ? !opening_check(pf.base_ef, root, l) : !opening_check(pf.base_bf, root, l))
      return false;
    for (unsigned k = 1; k < rounds; ++k)
      if (!opening_check(pf.folds[k - 1], pf.roots[k - 1], l >> k)) return false;
    auto val_at = [&](unsigned k, uint64_t p, ef2* v) -> bool {
      if (k == 0) return pf.leaf_ef ? base_value(pf.base_ef, p, eq4, v) : base_value(pf.base_bf, p, eq4, v);
      const auto& vals = pf.folds[k - 1].values;
      auto it = std::lower_bound(vals.begin(), vals.end(), p,
                                 [](const std::pair<uint64_t, std::vector<ef2>>& kv, uint64_t key) {
                                   return kv.first < key;
                                 });
      if (it == vals.end() || it->first != p || it->second.size() != 1) return false;
      *v = it->second[0];
      return true;
    };
    // fold consistency of every query down to the final codeword
    const uint64_t final_len = l >> rounds;
    for (uint64_t idx : base) {
      ef2 derived{};
      for (unsigned k = 0; k < rounds; ++k) {
        const uint64_t cur = l >> k, half = cur / 2, pos = idx % half, sib = pos + half;
        ef2 a, b;
        if (!val_at(k, pos, &a) || !val_at(k, sib, &b)) return false;
        if (k > 0 && !ef_eq(derived, (idx % cur == pos) ? a : b)) return false;
        derived = eq_fold_at(a, b, ch[k], cur, pos);
      }
      if (!ef_eq(derived, pf.final_codeword[idx % final_len])) return false;
    }
    // the final codeword is constant and equals the reduced claim
    for (const ef2& v : pf.final_codeword)
      if (!ef_eq(v, pf.final_codeword[0])) return false;
    return ef_eq(y, pf.final_codeword[0]);
  };
  bool ok;
  try {
    ok = run();
  } catch (const std::runtime_error&) {
    ok = false;  // oracle exhausted
  }
  cursors[0] = o.fi;
  cursors[1] = o.ii;
  return ok ? 1 : 0;
}

// Returns 1 accept, 0 reject.  Throws only on invalid arguments.
int verify_host(unsigned log_m, unsigned log_n, const Hash32& com_a, const Hash32& root,
                const u64* z_in, size_t zlen, const uint8_t* proof, size_t proof_len,
                const u64* fields, size_t nfields, const uint64_t* ints, size_t nints,
                uint64_t cursors[2]) {
  Shape s{log_m, log_n};
  if (!s.eval_ok()) throw std::invalid_argument("shape outside the shared-domain window");
  ProofH pf;
  if (!decode_proof(proof, proof_len, &pf)) return 0;
  if (zlen != log_m + log_n) return 0;
  Oracle o{fields, nfields, (size_t)cursors[0], ints, nints, (size_t)cursors[1]};
  const uint64_t n = s.n(), two_n = 2 * n, W = s.W(), S = NUM_COLS;
  EFv z(zlen);
  for (size_t i = 0; i < zlen; ++i) z[i] = ef_make(gl_canon(z_in[2 * i]), gl_canon(z_in[2 * i + 1]));
  EFv z2(z.begin(), z.begin() + log_n), z1(z.begin() + log_n, z.end());
  auto run = [&]() -> bool {
    auto eqz1 = new_eq(z1);
    std::vector<uint64_t> idx;
    if (!sample_columns(o.take_ints(4 * NUM_COLS), two_n, &idx)) return false;
    std::vector<uint64_t> sidx(idx);
    std::sort(sidx.begin(), sidx.end());
    if (pf.h_cols.size() != S) return false;
    for (auto& col : pf.h_cols)
      if (col.size() != DIGEST_ROWS) return false;
    {
      std::vector<Hash32> lh;
      for (auto& col : pf.h_cols) lh.push_back(hash_bytes(leaf_bytes(col)));
      if (!merkle_check(root, pf.h_open, sidx, lh, two_n)) return false;
    }
    {
      const unsigned log_w = s.log_w(), log_s = s.log_s();
      EFv alpha1 = o.fields(log_w + log_s), alpha2 = o.fields(5), ch;
      if (!sc_verify(ef_zero(), pf.sc[0], o, &ch)) return false;
      EFv r1 = rev(ch);
      auto& fe = pf.sc[0].finals;
      if (fe.size() != 3 || !ef_eq(fe[1], ef_sub(fe[0], ef_one())) || !ef_eq(fe[2], eval_eq(alpha1, r1)))
        return false;
      EFv r2 = o.fields(log_s);
      EFv eq_r2 = new_eq(r2), eq_a2 = new_eq(alpha2);
      ef2 y2 = ef_zero();
      for (size_t k = 0; k < S; ++k) {
        size_t pos = std::lower_bound(sidx.begin(), sidx.end(), idx[k]) - sidx.begin();
        ef2 t = ef_zero();
        for (unsigned r = 0; r < DIGEST_ROWS; ++r) t = ef_add(t, ef_scale(eq_a2[r], pf.h_cols[pos][r]));
        y2 = ef_add(y2, ef_mul(eq_r2[k], t));
      }
      if (!sc_verify(y2, pf.sc[1], o, &ch) || pf.sc[1].finals.size() != 2) return false;
      EFv r4 = rev(ch);
      if (!sc_verify(pf.y4, pf.sc[2], o, &ch)) return false;
      EFv r5 = rev(ch);
      {  // v(r5) with v[i] = eq_{z1}[i/64] 2^(i%64): separable over the low 6 bits
        EFv lo(r5.begin(), r5.begin() + 6), hi(r5.begin() + 6, r5.end());
        EFv el = new_eq(lo), eh = new_eq(hi);
        ef2 a = ef_zero(), b = ef_zero();
        for (unsigned q = 0; q < 64; ++q) a = ef_add(a, ef_scale(el[q], (u64)1 << q));
        for (size_t q = 0; q < eqz1.size(); ++q) b = ef_add(b, ef_mul(eqz1[q], eh[q]));
        if (pf.sc[2].finals.size() != 2 || !ef_eq(pf.sc[2].finals[0], ef_mul(a, b))) return false;
      }
      if (!sc_verify(pf.y4, pf.sc[3], o, &ch)) return false;
      EFv r3 = rev(ch);
      {  // sel(r3) = sum_k eq_r2[k] eq_{r3}(idx[k]) (sel is zero elsewhere)
        ef2 sv = ef_zero();
        for (size_t k = 0; k < S; ++k) {
          ef2 e = ef_one();
          for (size_t t = 0; t < r3.size(); ++t)
            e = ef_mul(e, ((idx[k] >> t) & 1) ? r3[t] : ef_sub(ef_one(), r3[t]));
          sv = ef_add(sv, ef_mul(eq_r2[k], e));
        }
        auto& f3 = pf.sc[3].finals;
        if (f3.size() != 2 || !ef_eq(f3[0], sv) || !ef_eq(f3[1], pf.y5)) return false;
      }
      if (!sc_verify(pf.y5, pf.sc[4], o, &ch)) return false;
      EFv r6 = rev(ch);
      {  // w(r6), w[k] = prod_t (1 - r3[t] + r3[t] g^((2^t k) mod 2n))
        const unsigned lg = ilog2_u64(two_n);
        const u64 g = gl_two_adic_generator(lg);
        std::vector<u64> gt(two_n);  // g^e for e < 2n
        gt[0] = 1;
        for (uint64_t e = 1; e < two_n; ++e) gt[e] = gl_mul(gt[e - 1], g);
        EFv w(n);
        for (uint64_t k = 0; k < n; ++k) {
          ef2 prod = ef_one();
          for (unsigned t = 0; t < lg; ++t) {
            u64 gv = gt[(k << t) & (two_n - 1)];
            prod = ef_mul(prod, ef_add(ef_sub(ef_one(), r3[t]), ef_scale(r3[t], gv)));
          }
          w[k] = prod;
        }
        if (pf.sc[4].finals.size() != 2 || !ef_eq(pf.sc[4].finals[1], mle_eval(w, r6))) return false;
      }
      EFv p_a = cat(r4, alpha2), p_bih = cat(r2, r4), p_bir = cat(r2, r5);
      ef2 gbi = o.field();
      std::vector<EFv> bpts{r1, p_bih, p_bir};
      ef2 fvals[3] = {pf.sc[0].finals[0], pf.sc[1].finals[1], pf.sc[2].finals[1]};
      ef2 claim = ef_zero();
      for (int i = 2; i >= 0; --i) claim = ef_add(ef_mul(claim, gbi), fvals[i]);
      if (!sc_verify(claim, pf.sc[5], o, &ch)) return false;
      EFv r_bi = rev(ch);
      {
        ef2 acc = ef_zero(), g = ef_one();
        for (auto& p : bpts) acc = ef_add(acc, ef_mul(g, eval_eq(p, r_bi))), g = ef_mul(g, gbi);
        if (pf.sc[5].finals.size() != 2 || !ef_eq(pf.sc[5].finals[1], acc)) return false;
      }
      ef2 ga = o.field();
      if (pf.sc[4].finals.size() != 2) return false;
      ef2 claim_a = ef_add(ef_mul(pf.sc[4].finals[0], ga), pf.y);
      if (!sc_verify(claim_a, pf.sc[6], o, &ch)) return false;
      EFv r_a = rev(ch);
      {
        ef2 acc = ef_add(eval_eq(z2, r_a), ef_mul(ga, eval_eq(r6, r_a)));
        if (pf.sc[6].finals.size() != 2 || !ef_eq(pf.sc[6].finals[1], acc)) return false;
      }
      std::vector<Claim> bfc{{com_a, p_a, pf.sc[1].finals[0], s.li(s.na())},
                             {pf.com_i, r_bi, pf.sc[5].finals[0], s.li(s.nbi())}};
      std::vector<Claim> efc{{pf.com_a_vec, r_a, pf.sc[6].finals[0], s.li(s.naa())}};
      return batch_verify(bfc, efc, pf.batch, o);
    }
  };
  int result = 0;
  try {
    result = run() ? 1 : 0;
  } catch (const std::runtime_error&) {
    result = 0;
  }
  cursors[0] = o.fi;
  cursors[1] = o.ii;
  return result;
}

}  // namespace lgs
