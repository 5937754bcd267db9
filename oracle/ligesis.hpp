// ORACLE (test infrastructure only): SubsetSumHash (pcs/src/subset_sum.rs:19-79) and the LigeSIS
// PCS (pcs/src/ligesis.rs: setup :239-273, commit :277-325, sample_columns :329-345,
// prove :347-549, rs_weights :553-567, verify :569-756, horner/combine_eq_eval :760-777).
// Every debug_assert of the reference prover is a hard check here.
#pragma once
#include <algorithm>
#include <vector>

#include "basefold.hpp"

namespace orc {

constexpr unsigned ETA = 64;               // ligesis.rs:53
constexpr unsigned CODE_RATE = 1;          // ligesis.rs:56
constexpr unsigned NUM_COLS_OPENED = 128;  // ligesis.rs:59
constexpr unsigned C = 32;                 // subset_sum.rs:19

inline unsigned lg2(size_t x) {
  unsigned k = 0;
  while ((size_t(1) << k) < x) ++k;
  return k;
}

// ligesis.rs:175-203
inline void committed_vars(unsigned log_m, unsigned log_n, unsigned out[3]) {
  out[0] = lg2(C) + lg2(ETA) + log_m;                // Ā
  out[1] = lg2(ETA) + log_m + lg2(NUM_COLS_OPENED);  // B_I
  out[2] = log_n;                                    // ā
}
inline bool shape_ok(unsigned log_m, unsigned log_n) {
  unsigned v[3];
  committed_vars(log_m, log_n, v);
  unsigned mx = std::max({v[0], v[1], v[2]}), mn = std::min({v[0], v[1], v[2]});
  return mx - mn <= LOG_INTERLEAVE && (size_t(2) << log_n) >= NUM_COLS_OPENED;
}
inline unsigned batch_rounds(unsigned log_m, unsigned log_n) {
  unsigned v[3];
  committed_vars(log_m, log_n, v);
  return std::max({v[0], v[1], v[2]}) - LOG_INTERLEAVE;
}
inline unsigned shared_li(unsigned nv, unsigned log_m, unsigned log_n) {
  return nv - batch_rounds(log_m, log_n);
}

struct ProvingKey {
  std::vector<u64> A;  // C x W row-major: A[r*W + i]
  size_t width = 0;
  BasefoldState<u64> a_state;
  Hash com_a;
  unsigned log_m = 0, log_n = 0;
};
struct VerifyingKey {
  Hash com_a;
  unsigned log_m = 0, log_n = 0;
  size_t width = 0;
};
struct CommitData {
  std::vector<u64> f;   // m x n row-major
  std::vector<u64> cw;  // m x 2n row-major RS codeword F' (its bits are B)
  std::vector<u64> H;   // C x 2n row-major digest
  MerkleTree h_tree;
};
struct LigesisProof {
  EF y;
  Hash com_a_vec, com_i;
  EF y4, y5;
  std::vector<std::vector<u64>> h_cols;  // sorted queried columns, C entries each
  std::vector<uint8_t> h_open;
  SumcheckProof sc_binary, sc_hash, sc_recon, sc_table, sc_rslink, sc_bi_batch, sc_a_batch;
  BatchProof batch;
};

// subset_sum.rs:58-67 — H[r][j] = sum over set bits i of column j of A[r][i].
inline std::vector<u64> hash_columns(const std::vector<u64>& A, size_t W,
                                     const std::vector<u64>& cw, size_t m, size_t two_n) {
  std::vector<u64> H(C * two_n, 0);
  // The same sums with A read column-wise: AT[i][r] = A[r][i], so the C additions of one set
  // bit touch one contiguous run (the reference reads A[r][i] across its rows).
  std::vector<u64> AT(W * C);
  for (unsigned r = 0; r < C; ++r)
    for (size_t i = 0; i < W; ++i) AT[i * C + r] = A[r * W + i];
  parallel_ranges(two_n, [&](size_t lo, size_t hi) {  // columns are independent
    u64 acc[C];
    for (size_t j = lo; j < hi; ++j) {
      for (unsigned r = 0; r < C; ++r) acc[r] = 0;
      for (size_t i = 0; i < m; ++i) {
        u64 v = cw[i * two_n + j];
        while (v) {
          const unsigned k = (unsigned)__builtin_ctzll(v);
          v &= v - 1;
          const u64* a = &AT[(ETA * i + k) * C];
          for (unsigned r = 0; r < C; ++r) {  // add() without branches
            u64 t = acc[r] + a[r];
            t += (u64)(t < a[r]) * EPS;
            acc[r] = t - (u64)(t >= P) * P;
          }
        }
      }
      for (unsigned r = 0; r < C; ++r) H[r * two_n + j] = acc[r];
    }
  }, 64);
  return H;
}

inline void setup(unsigned log_m, unsigned log_n, const u64* A_in, ProvingKey* pk,
                  VerifyingKey* vk) {
  if (!shape_ok(log_m, log_n))
    throw std::runtime_error("batched LigeSIS needs the {A, B_I, a} var counts within LOG_INTERLEAVE");
  size_t m = size_t(1) << log_m, W = ETA * m;
  pk->A.assign(A_in, A_in + C * W);
  for (auto& x : pk->A) x = canon(x);
  pk->width = W;
  unsigned a_vars = lg2(C * W);
  // a_mle_flat (subset_sum.rs:73-79) is exactly the row-major A.
  pk->a_state = commit_on_domain<u64>(pk->A, CODE_RATE, shared_li(a_vars, log_m, log_n), &pk->com_a);
  pk->log_m = log_m;
  pk->log_n = log_n;
  vk->com_a = pk->com_a;
  vk->log_m = log_m;
  vk->log_n = log_n;
  vk->width = W;
}

// A key for commit alone: Ligesis::commit (ligesis.rs:277-325) takes any m x n; only setup's
// Basefold commitment of A (and prove) need the shared-domain window.
inline void setup_commit_only(unsigned log_m, unsigned log_n, const u64* A_in, ProvingKey* pk) {
  size_t m = size_t(1) << log_m, W = ETA * m;
  pk->A.assign(A_in, A_in + C * W);
  for (auto& x : pk->A) x = canon(x);
  pk->width = W;
  pk->log_m = log_m;
  pk->log_n = log_n;
}

inline void commit(const ProvingKey& pk, const u64* f, size_t len, CommitData* cd, Hash* root) {
  size_t m = size_t(1) << pk.log_m, n = size_t(1) << pk.log_n, two_n = 2 * n;
  if (len != m * n) throw std::runtime_error("commit: f length");
  cd->f.assign(f, f + len);
  for (auto& x : cd->f) x = canon(x);
  cd->cw.assign(m * two_n, 0);
  parallel_ranges(m, [&](size_t lo, size_t hi) {  // ligesis.rs:288-300, rows are independent
    std::vector<u64> row(two_n);
    for (size_t i = lo; i < hi; ++i) {
      std::fill(row.begin(), row.end(), 0);
      std::copy(cd->f.begin() + i * n, cd->f.begin() + (i + 1) * n, row.begin());
      dft_bf(row);
      std::copy(row.begin(), row.end(), cd->cw.begin() + i * two_n);
    }
  });
  cd->H = hash_columns(pk.A, pk.width, cd->cw, m, two_n);
  std::vector<Hash> lh(two_n);  // ligesis.rs:306-313
  parallel_ranges(two_n, [&](size_t lo, size_t hi) {
    std::vector<u64> col(C);
    for (size_t j = lo; j < hi; ++j) {
      for (unsigned r = 0; r < C; ++r) col[r] = cd->H[r * two_n + j];
      auto b = serialize_bf(col);
      lh[j] = hash_bytes(b.data(), b.size());
    }
  }, size_t(1) << 10);
  cd->h_tree = MerkleTree::from_leaf_hashes(std::move(lh));
  *root = cd->h_tree.root();
}

inline std::vector<size_t> sample_columns(Oracle& o, size_t two_n, size_t s) {
  auto raw = o.next_n_ints(s * 4);  // ligesis.rs:329-345
  std::vector<char> seen(two_n, 0);
  std::vector<size_t> idx;
  for (u64 v : raw) {
    size_t j = (size_t)(v % two_n);
    if (!seen[j]) {
      seen[j] = 1;
      idx.push_back(j);
      if (idx.size() == s) break;
    }
  }
  if (idx.size() != s) throw std::runtime_error("not enough distinct columns sampled from oracle");
  return idx;
}

inline std::vector<EF> combine_eq(const std::vector<std::vector<EF>>& pts, EF gamma) {
  size_t len = size_t(1) << pts[0].size();  // ligesis.rs:159-171
  std::vector<EF> out(len, ef_zero());
  EF g = ef_one();
  for (auto& p : pts) {
    auto e = new_eq(p);
    parallel_ranges(len, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; ++i) out[i] += g * e[i];
    }, size_t(1) << 15);
    g *= gamma;
  }
  return out;
}
inline EF horner(const std::vector<EF>& v, EF gamma) {
  EF acc = ef_zero();
  for (size_t i = v.size(); i-- > 0;) acc = acc * gamma + v[i];
  return acc;
}
inline EF combine_eq_eval(const std::vector<std::vector<EF>>& pts, EF gamma,
                          const std::vector<EF>& r) {
  EF acc = ef_zero(), g = ef_one();
  for (auto& p : pts) {
    acc += g * eval_eq(p, r);
    g *= gamma;
  }
  return acc;
}
inline std::vector<EF> rs_weights(const std::vector<EF>& r3, size_t n, size_t two_n) {
  unsigned lg = lg2(two_n);  // ligesis.rs:553-567
  u64 g = two_adic_generator(lg);
  std::vector<EF> w(n);
  parallel_ranges(n, [&](size_t lo, size_t hi) {
    for (size_t k = lo; k < hi; ++k) {
      EF prod = ef_one();
      for (unsigned t = 0; t < lg; ++t) {
        u64 e = (u64)((((u128)1 << t) * k) % two_n);
        prod *= ef_one() - r3[t] + r3[t] * lift(pow(g, e));
      }
      w[k] = prod;
    }
  }, size_t(1) << 10);
  return w;
}

inline LigesisProof prove(const ProvingKey& pk, const CommitData& cd, const std::vector<EF>& z,
                          Oracle& o) {
  unsigned log_m = pk.log_m, log_n = pk.log_n;
  size_t m = size_t(1) << log_m, n = size_t(1) << log_n, two_n = 2 * n;
  size_t W = ETA * m, s = NUM_COLS_OPENED;
  unsigned log_s = lg2(s), log_w = lg2(W);
  if (z.size() != log_m + log_n) throw std::runtime_error("prove: point size");
  auto check = [](bool c, const char* what) {
    if (!c) throw std::runtime_error(what);
  };
  std::vector<EF> z2(z.begin(), z.begin() + log_n), z1(z.begin() + log_n, z.end());
  auto eqz1 = new_eq(z1);
  LigesisProof pf;
  std::vector<EF> a_vec(n, ef_zero());  // ligesis.rs:372-379 (columns are independent)
  parallel_ranges(n, [&](size_t lo, size_t hi) {
    for (size_t i = 0; i < m; ++i)
      for (size_t j = lo; j < hi; ++j) a_vec[j] += eqz1[i] * cd.f[i * n + j];
  }, size_t(1) << 12);
  pf.y = mle_eval(a_vec, z2);
  auto a_vec_state = commit_on_domain<EF>(a_vec, CODE_RATE, shared_li(log_n, log_m, log_n),
                                          &pf.com_a_vec);
  std::vector<EF> ra(a_vec);  // rs_encode_ext (ligesis.rs:225-229)
  ra.resize(two_n, ef_zero());
  dft_ef(ra);

  auto idx = sample_columns(o, two_n, s);
  std::vector<size_t> sorted_idx(idx);
  std::sort(sorted_idx.begin(), sorted_idx.end());
  pf.h_open = cd.h_tree.open(sorted_idx);
  for (size_t j : sorted_idx) {
    std::vector<u64> col(C);
    for (unsigned r = 0; r < C; ++r) col[r] = cd.H[r * two_n + j];
    pf.h_cols.push_back(col);
  }
  auto bit = [&](size_t i, size_t j) -> u64 {  // B[i][j] = bit i%64 of F'[i/64][j]
    return (cd.cw[(i / ETA) * two_n + j] >> (i % ETA)) & 1;
  };
  std::vector<u64> bi_flat(W * s);  // ligesis.rs:403-410
  parallel_ranges(W, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i)
      for (size_t k = 0; k < s; ++k) bi_flat[i * s + k] = bit(i, idx[k]);
  }, 256);
  unsigned bi_vars = lg2(W * s);
  auto bi_state = commit_on_domain<u64>(bi_flat, CODE_RATE, shared_li(bi_vars, log_m, log_n),
                                        &pf.com_i);

  auto alpha1 = o.next_n_fields(log_w + log_s);
  auto alpha2 = o.next_n_fields(lg2(C));
  auto eq_alpha2 = new_eq(alpha2);

  std::vector<EF> bi_ef(W * s), bi_m1(W * s);
  parallel_ranges(W * s, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) bi_ef[i] = lift(bi_flat[i]), bi_m1[i] = bi_ef[i] - ef_one();
  }, size_t(1) << 15);
  std::vector<EF> ch_bin;
  pf.sc_binary = sumcheck_prove({bi_ef, bi_m1, new_eq(alpha1)}, o, &ch_bin);
  auto r1 = rev(ch_bin);

  auto r2 = o.next_n_fields(log_s);
  auto eq_r2 = new_eq(r2);
  std::vector<EF> g1(W, ef_zero()), g2(W, ef_zero());
  for (size_t i = 0; i < W; ++i) {
    for (unsigned r = 0; r < C; ++r) g1[i] += eq_alpha2[r] * pk.A[r * W + i];
    for (size_t k = 0; k < s; ++k)
      if (bit(i, idx[k])) g2[i] += eq_r2[k];
  }
  pf.y4 = ef_zero();
  for (size_t k = 0; k < s; ++k) pf.y4 += eq_r2[k] * ra[idx[k]];
  {  // debug_assert ligesis.rs:461-471
    EF lhs = ef_zero(), rhs = ef_zero();
    for (size_t k = 0; k < s; ++k) {
      EF t = ef_zero();
      for (unsigned r = 0; r < C; ++r) t += eq_alpha2[r] * cd.H[r * two_n + idx[k]];
      lhs += eq_r2[k] * t;
    }
    for (size_t i = 0; i < W; ++i) rhs += g1[i] * g2[i];
    check(lhs == rhs, "prove: hash-channel identity");
  }
  std::vector<EF> v_vec(W);
  // pow2 (ligesis.rs:212-220): 2^k by repeated doubling; 2^k < p for k < 64, so it is 1 << k.
  for (size_t i = 0; i < W; ++i) v_vec[i] = eqz1[i / ETA] * lift(u64(1) << (i % ETA));
  {
    EF t = ef_zero();
    for (size_t i = 0; i < W; ++i) t += v_vec[i] * g2[i];
    check(t == pf.y4, "prove: recon identity");  // ligesis.rs:477
  }
  std::vector<EF> ch_hash, ch_recon, ch_table, ch_rs;
  pf.sc_hash = sumcheck_prove({g1, g2}, o, &ch_hash);
  auto r4 = rev(ch_hash);
  pf.sc_recon = sumcheck_prove({v_vec, g2}, o, &ch_recon);
  auto r5 = rev(ch_recon);
  std::vector<EF> sel(two_n, ef_zero());
  for (size_t k = 0; k < s; ++k) sel[idx[k]] = eq_r2[k];
  {
    EF t = ef_zero();
    for (size_t j = 0; j < two_n; ++j) t += sel[j] * ra[j];
    check(t == pf.y4, "prove: table identity");  // ligesis.rs:492
  }
  pf.sc_table = sumcheck_prove({sel, ra}, o, &ch_table);
  auto r3 = rev(ch_table);
  pf.y5 = mle_eval(ra, r3);
  auto w_vec = rs_weights(r3, n, two_n);
  {
    EF t = ef_zero();
    for (size_t k = 0; k < n; ++k) t += a_vec[k] * w_vec[k];
    check(t == pf.y5, "prove: rs-link identity");  // ligesis.rs:501
  }
  pf.sc_rslink = sumcheck_prove({a_vec, w_vec}, o, &ch_rs);
  auto p_a = cat(r4, alpha2);
  auto p_bi_hash = cat(r2, r4);
  auto p_bi_recon = cat(r2, r5);
  auto r6 = rev(ch_rs);

  EF gamma_bi = o.next_field();
  auto g_bi = combine_eq({r1, p_bi_hash, p_bi_recon}, gamma_bi);
  std::vector<EF> ch_bi, ch_a;
  pf.sc_bi_batch = sumcheck_prove({bi_ef, g_bi}, o, &ch_bi);
  auto r_bi = rev(ch_bi);
  EF gamma_a = o.next_field();
  auto g_a = combine_eq({z2, r6}, gamma_a);
  pf.sc_a_batch = sumcheck_prove({a_vec, g_a}, o, &ch_a);
  auto r_a = rev(ch_a);

  pf.batch = batch_prove({{&pk.a_state, p_a}, {&bi_state, r_bi}}, {{&a_vec_state, r_a}}, o);
  return pf;
}

inline bool verify(const VerifyingKey& vk, const Hash& commit, const std::vector<EF>& z,
                   const LigesisProof& pf, Oracle& o) {
  unsigned log_m = vk.log_m, log_n = vk.log_n;
  size_t m = size_t(1) << log_m, n = size_t(1) << log_n, two_n = 2 * n;
  size_t W = ETA * m, s = NUM_COLS_OPENED;
  unsigned log_s = lg2(s);
  if (z.size() != log_m + log_n) return false;
  std::vector<EF> z2(z.begin(), z.begin() + log_n), z1(z.begin() + log_n, z.end());
  auto eqz1 = new_eq(z1);
  auto idx = sample_columns(o, two_n, s);
  std::vector<size_t> sorted_idx(idx);
  std::sort(sorted_idx.begin(), sorted_idx.end());
  if (pf.h_cols.size() != sorted_idx.size()) return false;
  for (auto& c : pf.h_cols)
    if (c.size() != C) return false;
  std::vector<std::vector<uint8_t>> leaves;
  for (auto& c : pf.h_cols) leaves.push_back(serialize_bf(c));
  if (!merkle_verify(commit, pf.h_open, sorted_idx, leaves, two_n)) return false;

  auto alpha1 = o.next_n_fields(lg2(W) + log_s);
  auto alpha2 = o.next_n_fields(lg2(C));
  std::vector<EF> ch_bin;
  if (!sumcheck_verify(ef_zero(), pf.sc_binary, o, &ch_bin)) return false;
  auto r1 = rev(ch_bin);
  {
    auto& fe = pf.sc_binary.final_evals;
    if (fe.size() != 3 || fe[1] != fe[0] - ef_one() || fe[2] != eval_eq(alpha1, r1)) return false;
  }
  auto r2 = o.next_n_fields(log_s);
  auto eq_r2 = new_eq(r2);
  auto eq_alpha2 = new_eq(alpha2);
  EF y2 = ef_zero();
  for (size_t k = 0; k < s; ++k) {
    size_t pos = std::lower_bound(sorted_idx.begin(), sorted_idx.end(), idx[k]) - sorted_idx.begin();
    const auto& col = pf.h_cols[pos];
    EF t = ef_zero();
    for (unsigned r = 0; r < C; ++r) t += eq_alpha2[r] * lift(canon(col[r]));
    y2 += eq_r2[k] * t;
  }
  std::vector<EF> ch_hash, ch_recon, ch_table, ch_rs;
  if (!sumcheck_verify(y2, pf.sc_hash, o, &ch_hash)) return false;
  auto r4 = rev(ch_hash);
  if (pf.sc_hash.final_evals.size() != 2) return false;
  if (!sumcheck_verify(pf.y4, pf.sc_recon, o, &ch_recon)) return false;
  auto r5 = rev(ch_recon);
  std::vector<EF> v_vec(W);
  for (size_t i = 0; i < W; ++i) v_vec[i] = eqz1[i / ETA] * lift(u64(1) << (i % ETA));
  if (pf.sc_recon.final_evals.size() != 2 || pf.sc_recon.final_evals[0] != mle_eval(v_vec, r5))
    return false;
  if (!sumcheck_verify(pf.y4, pf.sc_table, o, &ch_table)) return false;
  auto r3 = rev(ch_table);
  std::vector<EF> sel(two_n, ef_zero());
  for (size_t k = 0; k < s; ++k) sel[idx[k]] = eq_r2[k];
  {
    auto& fe = pf.sc_table.final_evals;
    if (fe.size() != 2 || fe[0] != mle_eval(sel, r3) || fe[1] != pf.y5) return false;
  }
  if (!sumcheck_verify(pf.y5, pf.sc_rslink, o, &ch_rs)) return false;
  auto r6 = rev(ch_rs);
  auto w_vec = rs_weights(r3, n, two_n);
  if (pf.sc_rslink.final_evals.size() != 2 || pf.sc_rslink.final_evals[1] != mle_eval(w_vec, r6))
    return false;
  auto p_a = cat(r4, alpha2);
  auto p_bi_hash = cat(r2, r4);
  auto p_bi_recon = cat(r2, r5);
  EF gamma_bi = o.next_field();
  std::vector<std::vector<EF>> bi_pts{r1, p_bi_hash, p_bi_recon};
  EF claim_bi = horner({pf.sc_binary.final_evals[0], pf.sc_hash.final_evals[1],
                        pf.sc_recon.final_evals[1]},
                       gamma_bi);
  std::vector<EF> ch_bi, ch_a;
  if (!sumcheck_verify(claim_bi, pf.sc_bi_batch, o, &ch_bi)) return false;
  auto r_bi = rev(ch_bi);
  if (pf.sc_bi_batch.final_evals.size() != 2 ||
      pf.sc_bi_batch.final_evals[1] != combine_eq_eval(bi_pts, gamma_bi, r_bi))
    return false;
  EF v_bi = pf.sc_bi_batch.final_evals[0];
  EF gamma_a = o.next_field();
  std::vector<std::vector<EF>> a_pts{z2, r6};
  EF claim_a = horner({pf.y, pf.sc_rslink.final_evals[0]}, gamma_a);
  if (!sumcheck_verify(claim_a, pf.sc_a_batch, o, &ch_a)) return false;
  auto r_a = rev(ch_a);
  if (pf.sc_a_batch.final_evals.size() != 2 ||
      pf.sc_a_batch.final_evals[1] != combine_eq_eval(a_pts, gamma_a, r_a))
    return false;
  EF v_a = pf.sc_a_batch.final_evals[0];
  unsigned nv_a = lg2(C * W), nv_bi = lg2(W * s);
  std::vector<BatchClaim> bfc{{vk.com_a, p_a, pf.sc_hash.final_evals[0], shared_li(nv_a, log_m, log_n)},
                              {pf.com_i, r_bi, v_bi, shared_li(nv_bi, log_m, log_n)}};
  std::vector<BatchClaim> efc{{pf.com_a_vec, r_a, v_a, shared_li(log_n, log_m, log_n)}};
  return batch_verify(bfc, efc, pf.batch, o);
}

}  // namespace orc
