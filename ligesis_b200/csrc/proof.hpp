// Host-side LigeSIS proof structure (pcs/src/ligesis.rs:99-119; BatchProof of
// pcs/src/basefold.rs:151-162) and its byte encoding, plus the transcript index logic that the
// prover and the verifier share: column sampling (pcs/src/ligesis.rs:329-345), the shared
// FRI query set (pcs/src/basefold.rs:787-795), level positions (:234-244) and rs_merkle's
// multiproof node order (utils/src/merkle.rs:76-78).
//
// Encoding (all integers little-endian, BF = canonical u64, EF = c0 then c1, H32 = 32 bytes):
//   "LGSP" u32:1 | y:EF com_a_vec:H32 com_i:H32 y4:EF y5:EF
//   | h_cols: u32 ncols, u32 C, ncols*C BF | h_open: u32 nbytes, bytes
//   | 7 sumchecks (binary, hash, recon, table, rslink, bi_batch, a_batch), each
//       u32 rounds, u32 width, rounds*width EF, u32 nfinal, nfinal EF
//   | batch: u32 code_rate, u32 log_len, u32 nch, per channel (u32 len, len EF),
//       u32 nroots, H32*, u32 nfinal, EF*, u32 nfold, opening<EF>*, u32 nbf, opening<BF>*,
//       u32 nef, opening<EF>*
//   opening<F>: u32 nbytes, bytes, u32 nvals, per value (u64 key, u32 len, len F)
#pragma once
#include <algorithm>
#include <cstring>
#include <vector>

#include "gl64.cuh"

namespace lgs {

inline unsigned ilog2_u64(uint64_t x) {
  unsigned k = 0;
  while (((uint64_t)1 << k) < x) ++k;
  return k;
}

struct Hash32 {
  uint8_t b[32];
  bool operator==(const Hash32& o) const { return std::memcmp(b, o.b, 32) == 0; }
  bool operator!=(const Hash32& o) const { return !(*this == o); }
};

struct ScProof {
  std::vector<std::vector<ef2>> rounds;
  std::vector<ef2> finals;
};
template <class F>
struct OpeningH {
  std::vector<uint8_t> proof;
  std::vector<std::pair<uint64_t, std::vector<F>>> values;  // ascending keys
};
struct BatchProofH {
  std::vector<std::vector<ef2>> msgs;
  std::vector<Hash32> fold_roots;
  std::vector<ef2> final_codeword;
  std::vector<OpeningH<ef2>> fold_openings;
  std::vector<OpeningH<u64>> base_bf;
  std::vector<OpeningH<ef2>> base_ef;
  uint32_t code_rate = 0, log_len = 0;
};
struct ProofH {
  ef2 y, y4, y5;
  Hash32 com_a_vec, com_i;
  std::vector<std::vector<u64>> h_cols;
  std::vector<uint8_t> h_open;
  ScProof sc[7];
  BatchProofH batch;
};

// ---- protocol constants (pcs/src/ligesis.rs:53-59, pcs/src/subset_sum.rs:19,
// pcs/src/basefold.rs:15-16) and shape arithmetic (pcs/src/ligesis.rs:175-203) ----
constexpr unsigned ETA = 64, CODE_RATE = 1, NUM_COLS = 128, DIGEST_ROWS = 32,
                   LOG_INTERLEAVE = 6;
constexpr unsigned QUERIES = 100;  // ceil(100 / code_rate) at code_rate 1

struct Shape {
  unsigned log_m, log_n;
  unsigned log_w() const { return log_m + 6; }
  unsigned log_s() const { return 7; }
  unsigned na() const { return 5 + 6 + log_m; }
  unsigned nbi() const { return 6 + log_m + 7; }
  unsigned naa() const { return log_n; }
  unsigned vmax() const { return std::max(na(), std::max(nbi(), naa())); }
  unsigned vmin() const { return std::min(na(), std::min(nbi(), naa())); }
  // Ligesis::setup's shared-domain precondition (pcs/src/ligesis.rs:246-251).
  bool eval_ok() const { return vmax() - vmin() <= LOG_INTERLEAVE; }
  unsigned R() const { return vmax() - LOG_INTERLEAVE; }
  unsigned li(unsigned nv) const { return nv - R(); }
  size_t m() const { return (size_t)1 << log_m; }
  size_t n() const { return (size_t)1 << log_n; }
  size_t W() const { return (size_t)ETA << log_m; }
  size_t D() const { return (size_t)1 << (R() + CODE_RATE); }
};

// Oracle field offsets consumed by prove/verify, relative to the fields cursor on entry, in
// the order the reference draws them (pcs/src/ligesis.rs:419-530, pcs/src/basefold.rs:732-795).
struct FieldPlan {
  unsigned alpha1, alpha2, ch_bin, r2, ch_hash, ch_recon, ch_table, ch_rs, gamma_bi, ch_bi,
      gamma_a, ch_a, coeffs, ch_batch, total;
  explicit FieldPlan(const Shape& s) {
    unsigned nb = s.log_w() + s.log_s();
    alpha1 = 0;
    alpha2 = alpha1 + nb;
    ch_bin = alpha2 + 5;
    r2 = ch_bin + nb;
    ch_hash = r2 + s.log_s();
    ch_recon = ch_hash + s.log_w();
    ch_table = ch_recon + s.log_w();
    ch_rs = ch_table + s.log_n + 1;
    gamma_bi = ch_rs + s.log_n;
    ch_bi = gamma_bi + 1;
    gamma_a = ch_bi + nb;
    ch_a = gamma_a + 1;
    coeffs = ch_a + s.log_n;
    ch_batch = coeffs + 3;
    total = ch_batch + s.R();
  }
};
constexpr unsigned INTS_PER_PROOF = 4 * NUM_COLS + QUERIES;

// sample_columns: first s distinct values of ints mod 2n; false if fewer than s.  Seen values are
// kept in a small open-addressed set (at most 4s = 512 draws), not a 2n-entry table.
inline bool sample_columns(const uint64_t* ints, size_t two_n, std::vector<uint64_t>* idx) {
  constexpr unsigned SLOTS = 1024, EMPTY = ~0u;
  static_assert(SLOTS >= 2 * NUM_COLS, "set must stay at most half full");
  uint32_t slot[SLOTS];
  std::fill(slot, slot + SLOTS, EMPTY);
  idx->clear();
  for (unsigned t = 0; t < 4 * NUM_COLS; ++t) {
    const uint64_t j = ints[t] % two_n;
    unsigned h = (unsigned)((j * 0x9e3779b97f4a7c15ull) >> 54);  // 10-bit multiplicative hash
    bool fresh = true;
    while (slot[h] != EMPTY) {
      if ((*idx)[slot[h]] == j) {
        fresh = false;
        break;
      }
      h = (h + 1) & (SLOTS - 1);
    }
    if (fresh) {
      slot[h] = (uint32_t)idx->size();
      idx->push_back(j);
      if (idx->size() == NUM_COLS) return true;
    }
  }
  return false;
}
inline std::vector<uint64_t> query_base(const uint64_t* ints, size_t modulus) {
  std::vector<uint64_t> b;
  for (unsigned t = 0; t < QUERIES; ++t) b.push_back(ints[t] % modulus);
  std::sort(b.begin(), b.end());
  b.erase(std::unique(b.begin(), b.end()), b.end());
  return b;
}
inline std::vector<uint64_t> level_positions(const std::vector<uint64_t>& base, uint64_t half) {
  std::vector<uint64_t> p;
  for (uint64_t i : base) {
    p.push_back(i % half);
    p.push_back(i % half + half);
  }
  std::sort(p.begin(), p.end());
  p.erase(std::unique(p.begin(), p.end()), p.end());
  return p;
}
// Flat node indices (layer-major storage, leaves first) of the multiproof of sorted, distinct
// leaf indices in a power-of-two tree: per layer from the leaves up, the siblings that are not
// themselves known, ascending.
inline std::vector<uint64_t> multiproof_nodes(std::vector<uint64_t> cur, uint64_t leaves) {
  std::vector<uint64_t> out, par;
  uint64_t off = 0, len = leaves;
  while (len > 1) {
    par.clear();
    const size_t c = cur.size();
    for (size_t k = 0; k < c; ++k) {
      const uint64_t i = cur[k];
      // cur is sorted and distinct: i's sibling is known iff it is the neighbouring entry
      const bool known = (i & 1) ? (k > 0 && cur[k - 1] == i - 1) : (k + 1 < c && cur[k + 1] == i + 1);
      if (!known) out.push_back(off + (i ^ 1));
      if (par.empty() || par.back() != i / 2) par.push_back(i / 2);
    }
    cur.swap(par);
    off += len;
    len >>= 1;
  }
  return out;
}

// Upper bound on multiproof_nodes(q distinct leaves of a `leaves`-leaf tree): per layer at most
// one sibling per touched pair, and no more pairs than the layer has.
inline size_t multiproof_bound(uint64_t q, uint64_t leaves) {
  size_t total = 0;
  for (uint64_t len = leaves; len > 1; len >>= 1) {
    q = std::min<uint64_t>(q, len / 2);
    total += q;
  }
  return total;
}

// ---- encoding ----
struct ByteWriter {
  // Little-endian hosts only (x86-64, aarch64): integers are copied in memory order.
  static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "proof encoding assumes little-endian");
  // Writes into `b`, which only grows: a buffer reused across proofs is neither reallocated nor
  // cleared again once it is large enough.
  std::vector<uint8_t> own;
  std::vector<uint8_t>& b;
  size_t n = 0;
  ByteWriter() : b(own) {}
  explicit ByteWriter(std::vector<uint8_t>& into) : b(into) {}
  void need(size_t k) {
    if (n + k > b.size()) b.resize(std::max<size_t>(2 * b.size(), n + k + (1 << 16)));
  }
  void raw(const void* p, size_t k) {
    need(k);
    std::memcpy(b.data() + n, p, k);
    n += k;
  }
  void u32v(uint32_t v) { raw(&v, 4); }
  void u64v(uint64_t v) { raw(&v, 8); }
  // Shrinks the buffer to the bytes written and returns it (moved out of a writer that owns it).
  std::vector<uint8_t> finish() {
    b.resize(n);
    return std::move(b);
  }
  size_t finish_in_place() {
    b.resize(n);
    return n;
  }
  void bf(u64 v) { u64v(gl_canon(v)); }
  // `count` field elements from `src`, canonicalised (EF values are 2 consecutive words): one
  // bulk copy when every value is already canonical (a vectorisable check), else word by word.
  void bf_run(const u64* src, size_t count) {
    need(count * 8);
    uint8_t* d = b.data() + n;
    bool canon = true;
    for (size_t i = 0; i < count; ++i) canon &= src[i] < GL_P;
    if (canon) {
      std::memcpy(d, src, count * 8);
    } else {
      for (size_t i = 0; i < count; ++i) {
        const u64 v = gl_canon(src[i]);
        std::memcpy(d + 8 * i, &v, 8);
      }
    }
    n += count * 8;
  }
  void ef(const ef2& e) {
    bf(e.c0);
    bf(e.c1);
  }
  void h32(const Hash32& h) { raw(h.b, 32); }
  void bytes(const std::vector<uint8_t>& v) {
    u32v((uint32_t)v.size());
    raw(v.data(), v.size());
  }
  void val(u64 v) { bf(v); }
  void val(const ef2& v) { ef(v); }
  void sc(const ScProof& p) {
    u32v((uint32_t)p.rounds.size());
    u32v(p.rounds.empty() ? 0 : (uint32_t)p.rounds[0].size());
    for (auto& r : p.rounds)
      for (auto& e : r) ef(e);
    u32v((uint32_t)p.finals.size());
    for (auto& e : p.finals) ef(e);
  }
  template <class F>
  void opening(const OpeningH<F>& o) {
    bytes(o.proof);
    u32v((uint32_t)o.values.size());
    for (auto& kv : o.values) {
      u64v(kv.first);
      u32v((uint32_t)kv.second.size());
      for (auto& x : kv.second) val(x);
    }
  }
};

inline std::vector<uint8_t> encode_proof(const ProofH& p) {
  ByteWriter w;
  w.raw("LGSP", 4);
  w.u32v(1);
  w.ef(p.y);
  w.h32(p.com_a_vec);
  w.h32(p.com_i);
  w.ef(p.y4);
  w.ef(p.y5);
  w.u32v((uint32_t)p.h_cols.size());
  w.u32v(DIGEST_ROWS);
  for (auto& c : p.h_cols)
    for (u64 x : c) w.bf(x);
  w.bytes(p.h_open);
  for (int i = 0; i < 7; ++i) w.sc(p.sc[i]);
  const BatchProofH& b = p.batch;
  w.u32v(b.code_rate);
  w.u32v(b.log_len);
  w.u32v((uint32_t)b.msgs.size());
  for (auto& c : b.msgs) {
    w.u32v((uint32_t)c.size());
    for (auto& e : c) w.ef(e);
  }
  w.u32v((uint32_t)b.fold_roots.size());
  for (auto& h : b.fold_roots) w.h32(h);
  w.u32v((uint32_t)b.final_codeword.size());
  for (auto& e : b.final_codeword) w.ef(e);
  w.u32v((uint32_t)b.fold_openings.size());
  for (auto& o : b.fold_openings) w.opening(o);
  w.u32v((uint32_t)b.base_bf.size());
  for (auto& o : b.base_bf) w.opening(o);
  w.u32v((uint32_t)b.base_ef.size());
  for (auto& o : b.base_ef) w.opening(o);
  return w.finish();
}

struct ByteReader {
  const uint8_t* p;
  size_t n, pos = 0;
  bool ok = true;
  ByteReader(const uint8_t* d, size_t len) : p(d), n(len) {}
  bool need(size_t k) {
    if (!ok || pos > n || n - pos < k) ok = false;
    return ok;
  }
  uint32_t u32v() {
    if (!need(4)) return 0;
    uint32_t v = 0;
    for (int i = 0; i < 4; ++i) v |= (uint32_t)p[pos + i] << (8 * i);
    pos += 4;
    return v;
  }
  uint64_t u64v() {
    if (!need(8)) return 0;
    uint64_t v = 0;
    for (int i = 0; i < 8; ++i) v |= (uint64_t)p[pos + i] << (8 * i);
    pos += 8;
    return v;
  }
  u64 bf() {
    u64 v = u64v();
    if (v >= GL_P) ok = false;
    return v;
  }
  ef2 ef() {
    u64 a = bf();
    u64 b2 = bf();
    return ef_make(a, b2);
  }
  Hash32 h32() {
    Hash32 h{};
    if (!need(32)) return h;
    std::memcpy(h.b, p + pos, 32);
    pos += 32;
    return h;
  }
  std::vector<uint8_t> bytes() {
    uint32_t k = u32v();
    std::vector<uint8_t> v;
    if (!need(k)) return v;
    v.assign(p + pos, p + pos + k);
    pos += k;
    return v;
  }
  size_t count(size_t unit) {
    uint32_t k = u32v();
    if (ok && (size_t)k > (n - pos) / (unit ? unit : 1)) ok = false;
    return ok ? k : 0;
  }
  void val(u64* v) { *v = bf(); }
  void val(ef2* v) { *v = ef(); }
  ScProof sc() {
    ScProof s;
    uint32_t rounds = u32v(), width = u32v();
    if (!ok || rounds > 64 || width > 16) {
      ok = false;
      return s;
    }
    for (uint32_t r = 0; r < rounds && ok; ++r) {
      std::vector<ef2> e(width);
      for (uint32_t q = 0; q < width && ok; ++q) e[q] = ef();
      s.rounds.push_back(e);
    }
    size_t nf = count(16);
    for (size_t i = 0; i < nf && ok; ++i) s.finals.push_back(ef());
    return s;
  }
  template <class F>
  OpeningH<F> opening(size_t unit) {
    OpeningH<F> o;
    o.proof = bytes();
    size_t nv = count(12);
    for (size_t i = 0; i < nv && ok; ++i) {
      uint64_t key = u64v();
      if (i && key <= o.values.back().first) ok = false;
      size_t len = count(unit);
      std::vector<F> v(len);
      for (size_t j = 0; j < len && ok; ++j) val(&v[j]);
      o.values.push_back({key, v});
    }
    return o;
  }
};

// Standalone Basefold proof ("LGSB", pcs/src/basefold.rs:84-103):
//   "LGSB" u32:version=1, u32 num_vars, u32 code_rate, u32 log_interleave, u32 leaf_ef,
//   claimed_eval:EF, u32 rounds, rounds x (l0:EF, l1:EF), u32 nroots, nroots*H32,
//   u32 nfinal, nfinal EF, base opening<BF or EF>, u32 nfold, nfold*opening<EF>
struct BasefoldProofH {
  uint32_t num_vars = 0, code_rate = 0, log_interleave = 0, leaf_ef = 0;
  ef2 claimed{};
  std::vector<std::pair<ef2, ef2>> msgs;
  std::vector<Hash32> roots;
  std::vector<ef2> final_codeword;
  OpeningH<u64> base_bf;
  OpeningH<ef2> base_ef;
  std::vector<OpeningH<ef2>> folds;
};

inline bool decode_basefold_proof(const uint8_t* d, size_t len, BasefoldProofH* p) {
  ByteReader r(d, len);
  if (!r.need(4) || std::memcmp(d, "LGSB", 4) != 0) return false;
  r.pos = 4;
  if (r.u32v() != 1) return false;
  p->num_vars = r.u32v();
  p->code_rate = r.u32v();
  p->log_interleave = r.u32v();
  p->leaf_ef = r.u32v();
  if (!r.ok || p->num_vars > 40 || p->code_rate < 1 || p->code_rate > 8 ||
      p->log_interleave > 6 || p->log_interleave >= p->num_vars || p->leaf_ef > 1)
    return false;
  p->claimed = r.ef();
  size_t rounds = r.count(32);
  for (size_t i = 0; i < rounds && r.ok; ++i) {
    ef2 a = r.ef(), b = r.ef();
    p->msgs.push_back({a, b});
  }
  size_t nroots = r.count(32);
  for (size_t i = 0; i < nroots && r.ok; ++i) p->roots.push_back(r.h32());
  size_t nf = r.count(16);
  for (size_t i = 0; i < nf && r.ok; ++i) p->final_codeword.push_back(r.ef());
  if (p->leaf_ef)
    p->base_ef = r.opening<ef2>(16);
  else
    p->base_bf = r.opening<u64>(8);
  size_t nfo = r.count(8);
  for (size_t i = 0; i < nfo && r.ok; ++i) p->folds.push_back(r.opening<ef2>(16));
  return r.ok && r.pos == len;
}

inline bool decode_proof(const uint8_t* d, size_t len, ProofH* p) {
  ByteReader r(d, len);
  if (!r.need(4) || std::memcmp(d, "LGSP", 4) != 0) return false;
  r.pos = 4;
  if (r.u32v() != 1) return false;
  p->y = r.ef();
  p->com_a_vec = r.h32();
  p->com_i = r.h32();
  p->y4 = r.ef();
  p->y5 = r.ef();
  size_t ncols = r.count(8);
  uint32_t nrows = r.u32v();
  if (!r.ok || nrows > 1024) return false;
  p->h_cols.assign(ncols, std::vector<u64>(nrows));
  for (size_t i = 0; i < ncols && r.ok; ++i)
    for (uint32_t k = 0; k < nrows && r.ok; ++k) p->h_cols[i][k] = r.bf();
  p->h_open = r.bytes();
  for (int i = 0; i < 7; ++i) p->sc[i] = r.sc();
  BatchProofH& b = p->batch;
  b.code_rate = r.u32v();
  b.log_len = r.u32v();
  size_t nch = r.count(4);
  b.msgs.assign(nch, {});
  for (size_t c = 0; c < nch && r.ok; ++c) {
    size_t k = r.count(16);
    for (size_t i = 0; i < k && r.ok; ++i) b.msgs[c].push_back(r.ef());
  }
  size_t nroots = r.count(32);
  for (size_t i = 0; i < nroots && r.ok; ++i) b.fold_roots.push_back(r.h32());
  size_t nf = r.count(16);
  for (size_t i = 0; i < nf && r.ok; ++i) b.final_codeword.push_back(r.ef());
  size_t nfo = r.count(8);
  for (size_t i = 0; i < nfo && r.ok; ++i) b.fold_openings.push_back(r.opening<ef2>(16));
  size_t nbf = r.count(8);
  for (size_t i = 0; i < nbf && r.ok; ++i) b.base_bf.push_back(r.opening<u64>(8));
  size_t nef = r.count(8);
  for (size_t i = 0; i < nef && r.ok; ++i) b.base_ef.push_back(r.opening<ef2>(16));
  return r.ok && r.pos == len;
}

}  // namespace lgs
