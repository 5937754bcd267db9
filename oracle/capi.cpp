// ORACLE (test infrastructure only): C entry points over the CPU restatement, loaded by tests/
// through ctypes, by the smoke check and by bench.py's CPU-baseline leg.  Built into
// oracle/_build/liborc.so by oracle/Makefile.  Nothing in the product links this library.
//
// Buffers: BF = u64, EF = two u64 (c0, c1).  Status: 0 = ok, negative = error (message in
// orc_last_error()).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "frac_sum.hpp"
#include "proofsys.hpp"
#include "proof_io.hpp"

using namespace orc;

static thread_local std::string g_err;

#define ORC_TRY(...)                   \
  try {                                \
    __VA_ARGS__;                       \
  } catch (const std::exception& e) {  \
    g_err = e.what();                  \
    return -1;                         \
  }

static std::vector<EF> load_ef(const u64* p, size_t n) {
  std::vector<EF> v(n);
  for (size_t i = 0; i < n; ++i) v[i] = EF(p[2 * i], p[2 * i + 1]);
  return v;
}
static void store_ef(const EF& e, u64* out) {
  out[0] = e.c0;
  out[1] = e.c1;
}
static uint8_t* dup_bytes(const std::vector<uint8_t>& b, size_t* len) {
  uint8_t* p = (uint8_t*)std::malloc(b.size() ? b.size() : 1);
  if (!p) return nullptr;
  std::memcpy(p, b.data(), b.size());
  *len = b.size();
  return p;
}

struct OrcKey {
  ProvingKey pk;
  VerifyingKey vk;
};

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }
// Threads for the oracle's independent bulk loops (par.hpp); outputs do not depend on it.
void orc_set_threads(unsigned n) { oracle_threads() = n ? n : 1; }
unsigned orc_get_threads() { return oracle_threads(); }
void orc_free_buf(void* p) { std::free(p); }

// ---- field / primitive checks ----
int orc_two_adic_generator(unsigned bits, u64* out) { ORC_TRY(*out = two_adic_generator(bits)); return 0; }
int orc_bf_ops(const u64* a, const u64* b, size_t n, u64* sum, u64* diff, u64* prod) {
  for (size_t i = 0; i < n; ++i) {
    sum[i] = add(canon(a[i]), canon(b[i]));
    diff[i] = sub(canon(a[i]), canon(b[i]));
    prod[i] = mul(a[i], b[i]);
  }
  return 0;
}
int orc_ef_ops(const u64* a, const u64* b, size_t n, u64* prod, u64* inv_a) {
  ORC_TRY({
    for (size_t i = 0; i < n; ++i) {
      EF x(a[2 * i], a[2 * i + 1]), y(b[2 * i], b[2 * i + 1]);
      store_ef(x * y, prod + 2 * i);
      if (x != ef_zero()) store_ef(ef_inv(x), inv_a + 2 * i);
    }
  });
  return 0;
}
int orc_blake3(const uint8_t* data, size_t len, uint8_t* out) {
  Blake3::hash(data, len, out);
  return 0;
}
int orc_dft_bf(u64* data, size_t n) {
  ORC_TRY({
    std::vector<u64> v(data, data + n);
    dft_bf(v);
    std::memcpy(data, v.data(), n * 8);
  });
  return 0;
}
int orc_dft_ef(u64* data, size_t n) {
  ORC_TRY({
    auto v = load_ef(data, n);
    dft_ef(v);
    for (size_t i = 0; i < n; ++i) store_ef(v[i], data + 2 * i);
  });
  return 0;
}
int orc_mle_eval(const u64* evals, size_t k, const u64* point, u64* out) {
  ORC_TRY(store_ef(mle_eval(load_ef(evals, size_t(1) << k), load_ef(point, k)), out));
  return 0;
}
int orc_mle_fold(u64* evals, size_t k, const u64* point, size_t np) {
  ORC_TRY({
    auto v = load_ef(evals, size_t(1) << k);
    mle_fold(v, load_ef(point, np));
    for (size_t i = 0; i < v.size(); ++i) store_ef(v[i], evals + 2 * i);
  });
  return 0;
}
int orc_new_eq(const u64* point, size_t k, u64* out) {
  ORC_TRY({
    auto e = new_eq(load_ef(point, k));
    for (size_t i = 0; i < e.size(); ++i) store_ef(e[i], out + 2 * i);
  });
  return 0;
}
int orc_hash_columns(const u64* A, size_t W, const u64* cw, size_t m, size_t two_n, u64* H) {
  ORC_TRY({
    std::vector<u64> a(A, A + C * W), c(cw, cw + m * two_n);
    auto h = hash_columns(a, W, c, m, two_n);
    std::memcpy(H, h.data(), h.size() * 8);
  });
  return 0;
}
// d polys of 2^k EF each (poly-major); writes k*(d+1) round evals, d final evals, k challenges.
int orc_sumcheck_prove(const u64* polys, size_t d, size_t k, const u64* fields, size_t nf,
                       u64* rounds_out, u64* final_out, u64* ch_out) {
  ORC_TRY({
    std::vector<std::vector<EF>> ps;
    for (size_t j = 0; j < d; ++j) ps.push_back(load_ef(polys + 2 * j * (size_t(1) << k), size_t(1) << k));
    auto fv = load_ef(fields, nf);
    Oracle o;
    o.fields = fv.data();
    o.nfields = fv.size();
    std::vector<EF> ch;
    auto pf = sumcheck_prove(ps, o, &ch);
    for (size_t r = 0; r < pf.round_polys.size(); ++r)
      for (size_t t = 0; t <= d; ++t) store_ef(pf.round_polys[r][t], rounds_out + 2 * (r * (d + 1) + t));
    for (size_t j = 0; j < d; ++j) store_ef(pf.final_evals[j], final_out + 2 * j);
    for (size_t r = 0; r < ch.size(); ++r) store_ef(ch[r], ch_out + 2 * r);
  });
  return 0;
}
int orc_sumcheck_verify(const u64* claim, const u64* rounds_in, size_t k, size_t d,
                        const u64* final_in, const u64* fields, size_t nf) {
  ORC_TRY({
    SumcheckProof pf;
    for (size_t r = 0; r < k; ++r) pf.round_polys.push_back(load_ef(rounds_in + 2 * r * (d + 1), d + 1));
    pf.final_evals = load_ef(final_in, d);
    auto fv = load_ef(fields, nf);
    Oracle o;
    o.fields = fv.data();
    o.nfields = fv.size();
    std::vector<EF> ch;
    return sumcheck_verify(EF(claim[0], claim[1]), pf, o, &ch) ? 1 : 0;
  });
}
// leaves: n leaves of leaf_len bytes, contiguous.
int orc_merkle_root(const uint8_t* leaves, size_t n, size_t leaf_len, uint8_t* root) {
  std::vector<Hash> lh(n);
  for (size_t i = 0; i < n; ++i) lh[i] = hash_bytes(leaves + i * leaf_len, leaf_len);
  auto t = MerkleTree::from_leaf_hashes(std::move(lh));
  std::memcpy(root, t.root().data(), 32);
  return 0;
}
int orc_merkle_open(const uint8_t* leaves, size_t n, size_t leaf_len, const uint64_t* idx,
                    size_t nidx, uint8_t** out, size_t* out_len) {
  std::vector<Hash> lh(n);
  for (size_t i = 0; i < n; ++i) lh[i] = hash_bytes(leaves + i * leaf_len, leaf_len);
  auto t = MerkleTree::from_leaf_hashes(std::move(lh));
  std::vector<size_t> ix(idx, idx + nidx);
  *out = dup_bytes(t.open(ix), out_len);
  return 0;
}
int orc_merkle_verify(const uint8_t* root, const uint8_t* proof, size_t proof_len,
                      const uint64_t* idx, size_t nidx, const uint8_t* leaves, size_t leaf_len,
                      size_t total) {
  std::vector<size_t> ix(idx, idx + nidx);
  std::vector<std::vector<uint8_t>> lv;
  for (size_t i = 0; i < nidx; ++i) lv.emplace_back(leaves + i * leaf_len, leaves + (i + 1) * leaf_len);
  Hash r;
  std::memcpy(r.data(), root, 32);
  return merkle_verify(r, std::vector<uint8_t>(proof, proof + proof_len), ix, lv, total) ? 1 : 0;
}

// ---- LigeSIS ----
int orc_shape_ok(unsigned log_m, unsigned log_n) { return shape_ok(log_m, log_n) ? 1 : 0; }
void* orc_setup(unsigned log_m, unsigned log_n, const u64* A, uint8_t* com_a) {
  try {
    auto* k = new OrcKey;
    setup(log_m, log_n, A, &k->pk, &k->vk);
    std::memcpy(com_a, k->pk.com_a.data(), 32);
    return k;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void* orc_setup_commit_only(unsigned log_m, unsigned log_n, const u64* A) {
  try {
    auto* k = new OrcKey;
    setup_commit_only(log_m, log_n, A, &k->pk);
    return k;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void orc_key_free(void* k) { delete (OrcKey*)k; }
void* orc_commit(void* key, const u64* f, size_t len, uint8_t* root) {
  try {
    auto* cd = new CommitData;
    Hash h;
    commit(((OrcKey*)key)->pk, f, len, cd, &h);
    std::memcpy(root, h.data(), 32);
    return cd;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void orc_commit_free(void* cd) { delete (CommitData*)cd; }
int orc_commit_codeword(void* cd, u64* out) {
  auto* c = (CommitData*)cd;
  std::memcpy(out, c->cw.data(), c->cw.size() * 8);
  return 0;
}
int orc_commit_digest(void* cd, u64* out) {
  auto* c = (CommitData*)cd;
  std::memcpy(out, c->H.data(), c->H.size() * 8);
  return 0;
}
// cursors[0..2] = (fields, ints) consumed so far, in/out.
int orc_prove(void* key, void* cd, const u64* z, size_t zlen, const u64* fields, size_t nf,
              const u64* ints, size_t ni, uint64_t* cursors, uint8_t** proof, size_t* proof_len) {
  ORC_TRY({
    auto fv = load_ef(fields, nf);
    Oracle o;
    o.fields = fv.data();
    o.nfields = fv.size();
    o.ints = ints;
    o.nints = ni;
    o.fi = cursors[0];
    o.ii = cursors[1];
    auto pf = prove(((OrcKey*)key)->pk, *(CommitData*)cd, load_ef(z, zlen), o);
    cursors[0] = o.fi;
    cursors[1] = o.ii;
    *proof = dup_bytes(encode_proof(pf), proof_len);
  });
  return 0;
}
int orc_verify(const uint8_t* com_a, unsigned log_m, unsigned log_n, const uint8_t* root,
               const u64* z, size_t zlen, const uint8_t* proof, size_t proof_len,
               const u64* fields, size_t nf, const u64* ints, size_t ni, uint64_t* cursors) {
  ORC_TRY({
    LigesisProof pf;
    if (!decode_proof(proof, proof_len, &pf)) return 0;
    VerifyingKey vk;
    std::memcpy(vk.com_a.data(), com_a, 32);
    vk.log_m = log_m;
    vk.log_n = log_n;
    vk.width = (size_t)ETA << log_m;
    Hash r;
    std::memcpy(r.data(), root, 32);
    auto fv = load_ef(fields, nf);
    Oracle o;
    o.fields = fv.data();
    o.nfields = fv.size();
    o.ints = ints;
    o.nints = ni;
    o.fi = cursors[0];
    o.ii = cursors[1];
    bool okv;
    try {
      okv = verify(vk, r, load_ef(z, zlen), pf, o);
    } catch (const std::exception&) {
      okv = false;  // e.g. oracle exhausted by a malformed proof's shape
    }
    cursors[0] = o.fi;
    cursors[1] = o.ii;
    return okv ? 1 : 0;
  });
}

// ---- standalone Basefold (pcs/src/basefold.rs:309-642) ----
struct OrcBasefold {
  int is_ef = 0;
  BasefoldState<u64> bf;
  BasefoldState<EF> ef;
};
void* orc_basefold_commit(const u64* poly, size_t len, int is_ef, unsigned code_rate, unsigned li,
                          uint8_t* root) {
  try {
    auto* h = new OrcBasefold;
    h->is_ef = is_ef;
    Hash r;
    if (is_ef) {
      h->ef = commit_on_domain(load_ef(poly, len), code_rate, li, &r);
    } else {
      std::vector<u64> v(poly, poly + len);
      for (auto& x : v) x = canon(x);
      h->bf = commit_on_domain(v, code_rate, li, &r);
    }
    std::memcpy(root, r.data(), 32);
    return h;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void orc_basefold_free(void* h) { delete (OrcBasefold*)h; }
int orc_basefold_prove(void* h, const u64* point, size_t plen, const u64* fields, size_t nf,
                       const u64* ints, size_t ni, uint64_t* cursors, uint8_t** proof,
                       size_t* proof_len) {
  ORC_TRY({
    auto fv = load_ef(fields, nf);
    Oracle o;
    o.fields = fv.data();
    o.nfields = fv.size();
    o.ints = ints;
    o.nints = ni;
    o.fi = cursors[0];
    o.ii = cursors[1];
    auto* b = (OrcBasefold*)h;
    const auto pt = load_ef(point, plen);
    std::vector<uint8_t> bytes = b->is_ef ? encode_basefold_proof(basefold_prove(b->ef, pt, o))
                                          : encode_basefold_proof(basefold_prove(b->bf, pt, o));
    cursors[0] = o.fi;
    cursors[1] = o.ii;
    *proof = dup_bytes(bytes, proof_len);
  });
  return 0;
}
int orc_basefold_verify(const uint8_t* root, const u64* point, size_t plen, const uint8_t* proof,
                        size_t proof_len, const u64* fields, size_t nf, const u64* ints,
                        size_t ni, uint64_t* cursors) {
  ORC_TRY({
    const int leaf_ef = basefold_proof_leaf_ef(proof, proof_len);
    if (leaf_ef < 0) return 0;
    Hash r;
    std::memcpy(r.data(), root, 32);
    auto fv = load_ef(fields, nf);
    Oracle o;
    o.fields = fv.data();
    o.nfields = fv.size();
    o.ints = ints;
    o.nints = ni;
    o.fi = cursors[0];
    o.ii = cursors[1];
    const auto pt = load_ef(point, plen);
    bool okv = false;
    try {
      if (leaf_ef) {
        BasefoldProof<EF> pf;
        okv = decode_basefold_proof(proof, proof_len, &pf) && basefold_verify(r, pt, pf, o);
      } else {
        BasefoldProof<u64> pf;
        okv = decode_basefold_proof(proof, proof_len, &pf) && basefold_verify(r, pt, pf, o);
      }
    } catch (const std::exception&) {
      okv = false;
    }
    cursors[0] = o.fi;
    cursors[1] = o.ii;
    return okv ? 1 : 0;
  });
}

}  // extern "C"

// ---- GKR fraction sum and GKR-LogUp lookup (logup/src/frac_sum.rs, logup/src/lookup.rs) -----
static Oracle make_oracle(const std::vector<EF>& fv, const u64* ints, size_t ni,
                          const uint64_t* cursors) {
  Oracle o;
  o.fields = fv.data();
  o.nfields = fv.size();
  o.ints = ints;
  o.nints = ni;
  o.fi = cursors[0];
  o.ii = cursors[1];
  return o;
}
static void store_claim(const FsClaim& c, u64* point, u64* pq) {
  for (size_t i = 0; i < c.point.size(); ++i) store_ef(c.point[i], point + 2 * i);
  store_ef(c.p, pq);
  store_ef(c.q, pq + 2);
}

extern "C" {
// p == NULL: the numerators are all one.  point receives log2(n) EF, pq receives p_in(point) and
// q_in(point).
int orc_frac_sum_prove(const u64* p, const u64* q, size_t n, const u64* fields, size_t nf,
                       uint64_t* cursors, uint8_t** proof, size_t* proof_len, u64* point,
                       u64* pq) {
  ORC_TRY({
    auto fv = load_ef(fields, nf);
    Oracle o = make_oracle(fv, nullptr, 0, cursors);
    std::vector<EF> pv = p ? load_ef(p, n) : std::vector<EF>(n, ef_one());
    FsClaim c;
    auto pf = frac_sum_prove(pv, load_ef(q, n), o, &c);
    cursors[0] = o.fi;
    store_claim(c, point, pq);
    *proof = dup_bytes(encode_frac_sum_proof(pf), proof_len);
  });
  return 0;
}
// 1 accept, 0 reject; point receives nlayers EF.
int orc_frac_sum_verify(const uint8_t* proof, size_t len, const u64* fields, size_t nf,
                        uint64_t* cursors, u64* point, size_t point_cap, u64* pq) {
  ORC_TRY({
    FracSumProof pf;
    if (!decode_frac_sum_proof(proof, len, &pf) || pf.layers.size() > point_cap) return 0;
    auto fv = load_ef(fields, nf);
    Oracle o = make_oracle(fv, nullptr, 0, cursors);
    FsClaim c;
    bool okv = false;
    try {
      okv = frac_sum_verify(pf, o, &c);
    } catch (const std::exception&) {
      okv = false;
    }
    cursors[0] = o.fi;
    if (!okv) return 0;
    store_claim(c, point, pq);
  });
  return 1;
}
// e == NULL: the multiplicities are counted from a and t (lookup.rs:85-88).
int orc_lookup_prove(const u64* a, size_t m, const u64* t, size_t n, const u64* e,
                     const u64* fields, size_t nf, uint64_t* cursors, uint8_t** proof,
                     size_t* proof_len, u64* zq, u64* zt) {
  ORC_TRY({
    auto fv = load_ef(fields, nf);
    Oracle o = make_oracle(fv, nullptr, 0, cursors);
    auto av = load_ef(a, m), tv = load_ef(t, n);
    auto ev = e ? load_ef(e, n) : lookup_multiplicities(av, tv);
    std::vector<EF> pq, pt;
    auto pf = lookup_prove(av, tv, ev, o, &pq, &pt);
    cursors[0] = o.fi;
    for (size_t i = 0; i < pq.size(); ++i) store_ef(pq[i], zq + 2 * i);
    for (size_t i = 0; i < pt.size(); ++i) store_ef(pt[i], zt + 2 * i);
    *proof = dup_bytes(encode_lookup_proof(pf), proof_len);
  });
  return 0;
}
// 1 accept, 0 reject.  vals receives a(zq), e(zt), t(zt); zq / zt receive the points (their
// lengths are the proof's layer counts, at most the given capacities).
int orc_lookup_verify(const uint8_t* proof, size_t len, const u64* fields, size_t nf,
                      uint64_t* cursors, u64* zq, size_t zq_cap, u64* zt, size_t zt_cap,
                      u64* vals) {
  ORC_TRY({
    LookupProof pf;
    if (!decode_lookup_proof(proof, len, &pf) || pf.query.layers.size() > zq_cap ||
        pf.table.layers.size() > zt_cap)
      return 0;
    auto fv = load_ef(fields, nf);
    Oracle o = make_oracle(fv, nullptr, 0, cursors);
    LookupClaims c;
    bool okv = false;
    try {
      okv = lookup_verify(pf, o, &c);
    } catch (const std::exception&) {
      okv = false;
    }
    cursors[0] = o.fi;
    if (!okv) return 0;
    for (size_t i = 0; i < c.zq.size(); ++i) store_ef(c.zq[i], zq + 2 * i);
    for (size_t i = 0; i < c.zt.size(); ++i) store_ef(c.zt[i], zt + 2 * i);
    store_ef(c.a, vals);
    store_ef(c.e, vals + 2);
    store_ef(c.t, vals + 4);
  });
  return 1;
}

// proofsys' rescaled linear-layer witness (proofsys/src/tensor.rs, model.rs:360-361); bias may be
// NULL, y_field (encode_i64 of y) may be NULL.
int orc_linear_witness(const int64_t* x, size_t rows, size_t inner, const int64_t* w, size_t cols,
                       int w_transposed, const int64_t* bias, int64_t divisor, int64_t* q,
                       int64_t* rem, int64_t* y, uint64_t* y_field) {
  ORC_TRY({
    std::vector<i64> xv(x, x + rows * inner), wv(w, w + inner * cols), bv;
    if (bias) bv.assign(bias, bias + cols);
    const LinearWitness lw =
        linear_witness(xv, rows, inner, wv, cols, w_transposed != 0, bias ? &bv : nullptr, divisor);
    for (size_t i = 0; i < rows * cols; ++i) {
      q[i] = lw.q[i];
      rem[i] = lw.rem[i];
      y[i] = lw.y[i];
      if (y_field) y_field[i] = encode_i64(lw.y[i]);
    }
  });
  return 0;
}

// proofsys' layer-norm witness (proofsys/src/model.rs:241-279); per-row outputs hold rows values,
// per-entry outputs rows x d.
int orc_layer_norm_witness(const int64_t* x, size_t rows, size_t d, const int64_t* gain,
                           const int64_t* bias, int64_t* sum_x, int64_t* sum_x2, int64_t* var_sum,
                           int64_t* stdv, int64_t* dividend, int64_t* quotient, int64_t* output) {
  ORC_TRY({
    const LayerNormWitness w = layer_norm_witness(std::vector<i64>(x, x + rows * d), rows, d,
                                                  std::vector<i64>(gain, gain + d),
                                                  std::vector<i64>(bias, bias + d));
    std::copy(w.sum_x.begin(), w.sum_x.end(), sum_x);
    std::copy(w.sum_x2.begin(), w.sum_x2.end(), sum_x2);
    std::copy(w.var_sum.begin(), w.var_sum.end(), var_sum);
    std::copy(w.stdv.begin(), w.stdv.end(), stdv);
    std::copy(w.dividend.begin(), w.dividend.end(), dividend);
    std::copy(w.quotient.begin(), w.quotient.end(), quotient);
    std::copy(w.output.begin(), w.output.end(), output);
  });
  return 0;
}

// One GPT-2 block's witness (see block_witness): dims = n, d, heads, d_head, hidden; consts =
// scale, sqrt_d_scale, offset; weights in BlockWeights order; out receives the 36 arrays.
int orc_block_witness(const int64_t* x, const uint64_t* dims, const int64_t* consts,
                      const int64_t* const* weights, const int64_t* exp_lut, size_t exp_len,
                      const int64_t* gelu_lut, size_t gelu_len, int64_t* const* out) {
  ORC_TRY({
    GptDims g{dims[0], dims[1], dims[2], dims[3], dims[4], consts[0], consts[1], consts[2]};
    const size_t n = g.n, d = g.d, hid = g.hidden;
    const size_t sizes[12] = {d, d, d * 3 * d, 3 * d, d * d, d, d, d, d * hid, hid, hid * d, d};
    BlockWeights w;
    std::vector<i64>* fields[12] = {&w.ln1_g, &w.ln1_b, &w.attn_w, &w.attn_b, &w.proj_w,
                                    &w.proj_b, &w.ln2_g, &w.ln2_b, &w.fc_w, &w.fc_b, &w.fproj_w,
                                    &w.fproj_b};
    for (int i = 0; i < 12; ++i) fields[i]->assign(weights[i], weights[i] + sizes[i]);
    const auto res = block_witness(std::vector<i64>(x, x + n * d), g, w,
                                   std::vector<i64>(exp_lut, exp_lut + exp_len),
                                   std::vector<i64>(gelu_lut, gelu_lut + gelu_len));
    for (size_t i = 0; i < res.size(); ++i) std::copy(res[i].begin(), res[i].end(), out[i]);
  });
  return 0;
}
}  // extern "C"
