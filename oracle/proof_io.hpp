// ORACLE (test infrastructure only): byte encoding of a LigesisProof (field order of
// pcs/src/ligesis.rs:99-119, BatchProof of pcs/src/basefold.rs:151-162).  The reference keeps
// proofs as Rust structs and never serializes them, so this layout is the boundary's own; the
// product library writes the identical layout and the parity tests compare the bytes.
//
//   "LGSP" u32:version=1
//   y:EF com_a_vec:H32 com_i:H32 y4:EF y5:EF
//   h_cols: u32 ncols, u32 C, ncols*C BF (column by column, columns in sorted index order)
//   h_open: u32 nbytes, bytes
//   7 x sumcheck (binary, hash, recon, table, rslink, bi_batch, a_batch):
//        u32 rounds, u32 width(d+1), rounds*width EF, u32 nfinal, nfinal EF
//   batch: u32 code_rate, u32 log_len,
//          u32 nch, per channel (u32 len, len EF),
//          u32 nroots, nroots*H32, u32 nfinal, nfinal EF,
//          u32 nfold, nfold*opening<EF>, u32 nbf, nbf*opening<BF>, u32 nef, nef*opening<EF>
//   opening<F>: u32 nbytes, bytes, u32 nvals, per value (u64 key, u32 len, len F), keys ascending
// Integers are little-endian; BF is a canonical u64; EF is c0 then c1.
//
// Standalone BasefoldProof (pcs/src/basefold.rs:84-103), the same conventions:
//   "LGSB" u32:version=1
//   u32 num_vars, u32 code_rate, u32 log_interleave, u32 leaf_ef (0: BF leaves, 1: EF leaves)
//   claimed_eval:EF, u32 rounds, rounds x (l0:EF, l1:EF)
//   u32 nroots, nroots*H32, u32 nfinal, nfinal EF
//   base:opening<LF>, u32 nfold, nfold*opening<EF>
#pragma once
#include <cstring>
#include <vector>

#include "ligesis.hpp"

namespace orc {

struct Writer {
  std::vector<uint8_t> b;
  void u32(uint32_t v) {
    for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i)));
  }
  void u64v(u64 v) { ser_u64(b, v); }
  void bf(u64 v) { ser_u64(b, canon(v)); }
  void ef(const EF& e) {
    bf(e.c0);
    bf(e.c1);
  }
  void hash(const Hash& h) { b.insert(b.end(), h.begin(), h.end()); }
  void bytes(const std::vector<uint8_t>& v) {
    u32((uint32_t)v.size());
    b.insert(b.end(), v.begin(), v.end());
  }
  void sc(const SumcheckProof& p) {
    u32((uint32_t)p.round_polys.size());
    u32(p.round_polys.empty() ? 0 : (uint32_t)p.round_polys[0].size());
    for (auto& r : p.round_polys)
      for (auto& e : r) ef(e);
    u32((uint32_t)p.final_evals.size());
    for (auto& e : p.final_evals) ef(e);
  }
  void val(u64 v) { bf(v); }
  void val(const EF& v) { ef(v); }
  template <class F>
  void opening(const Opening<F>& op) {
    bytes(op.proof_bytes);
    u32((uint32_t)op.values.size());
    for (auto& kv : op.values) {
      u64v(kv.first);
      u32((uint32_t)kv.second.size());
      for (auto& x : kv.second) val(x);
    }
  }
};

inline std::vector<uint8_t> encode_proof(const LigesisProof& p) {
  Writer w;
  w.b.insert(w.b.end(), {'L', 'G', 'S', 'P'});
  w.u32(1);
  w.ef(p.y);
  w.hash(p.com_a_vec);
  w.hash(p.com_i);
  w.ef(p.y4);
  w.ef(p.y5);
  w.u32((uint32_t)p.h_cols.size());
  w.u32(C);
  for (auto& c : p.h_cols)
    for (u64 x : c) w.bf(x);
  w.bytes(p.h_open);
  for (const SumcheckProof* s : {&p.sc_binary, &p.sc_hash, &p.sc_recon, &p.sc_table, &p.sc_rslink,
                                 &p.sc_bi_batch, &p.sc_a_batch})
    w.sc(*s);
  const BatchProof& b = p.batch;
  w.u32(b.code_rate);
  w.u32(b.log_len);
  w.u32((uint32_t)b.reduction_msgs.size());
  for (auto& ch : b.reduction_msgs) {
    w.u32((uint32_t)ch.size());
    for (auto& e : ch) w.ef(e);
  }
  w.u32((uint32_t)b.fold_roots.size());
  for (auto& h : b.fold_roots) w.hash(h);
  w.u32((uint32_t)b.final_codeword.size());
  for (auto& e : b.final_codeword) w.ef(e);
  w.u32((uint32_t)b.fold_openings.size());
  for (auto& o : b.fold_openings) w.opening(o);
  w.u32((uint32_t)b.base_bf.size());
  for (auto& o : b.base_bf) w.opening(o);
  w.u32((uint32_t)b.base_ef.size());
  for (auto& o : b.base_ef) w.opening(o);
  return w.b;
}

// Bounds-checked decoder; any malformed input yields false (never a crash).
struct Reader {
  const uint8_t* p;
  size_t n, pos = 0;
  bool ok = true;
  Reader(const uint8_t* d, size_t len) : p(d), n(len) {}
  bool need(size_t k) {
    if (!ok || n - pos < k || pos > n) ok = false;
    return ok;
  }
  uint32_t u32() {
    if (!need(4)) return 0;
    uint32_t v = 0;
    for (int i = 0; i < 4; ++i) v |= (uint32_t)p[pos + i] << (8 * i);
    pos += 4;
    return v;
  }
  u64 u64v() {
    if (!need(8)) return 0;
    u64 v = 0;
    for (int i = 0; i < 8; ++i) v |= (u64)p[pos + i] << (8 * i);
    pos += 8;
    return v;
  }
  // Non-canonical field encodings are rejected (a canonical encoder never writes them).
  u64 bf() {
    u64 v = u64v();
    if (v >= P) ok = false;
    return v;
  }
  EF ef() {
    u64 a = bf(), b = bf();
    return EF(a, b);
  }
  Hash hash() {
    Hash h{};
    if (!need(32)) return h;
    std::memcpy(h.data(), p + pos, 32);
    pos += 32;
    return h;
  }
  std::vector<uint8_t> bytes() {
    uint32_t k = u32();
    std::vector<uint8_t> v;
    if (!need(k)) return v;
    v.assign(p + pos, p + pos + k);
    pos += k;
    return v;
  }
  size_t count(size_t unit) {  // a u32 count whose payload must fit in what is left
    uint32_t k = u32();
    if (ok && (unit ? (size_t)k > (n - pos) / unit : k > (1u << 24))) ok = false;
    return ok ? k : 0;
  }
  SumcheckProof sc() {
    SumcheckProof s;
    size_t rounds = u32(), width = u32();
    if (!ok || rounds > 64 || width > 16) {
      ok = false;
      return s;
    }
    for (size_t r = 0; r < rounds && ok; ++r) {
      std::vector<EF> ev;
      for (size_t k = 0; k < width && ok; ++k) ev.push_back(ef());
      s.round_polys.push_back(ev);
    }
    size_t nf = count(16);
    for (size_t i = 0; i < nf && ok; ++i) s.final_evals.push_back(ef());
    return s;
  }
  void val(u64* v) { *v = bf(); }
  void val(EF* v) { *v = ef(); }
  template <class F>
  Opening<F> opening(size_t unit) {
    Opening<F> op;
    op.proof_bytes = bytes();
    size_t nv = count(12);
    u64 last = 0;
    for (size_t i = 0; i < nv && ok; ++i) {
      u64 key = u64v();
      if (i && key <= last) ok = false;
      last = key;
      size_t len = count(unit);
      std::vector<F> vals(len);
      for (size_t j = 0; j < len && ok; ++j) val(&vals[j]);
      op.values[(size_t)key] = vals;
    }
    return op;
  }
};

inline bool decode_proof(const uint8_t* data, size_t len, LigesisProof* p) {
  Reader r(data, len);
  if (!r.need(4) || std::memcmp(data, "LGSP", 4) != 0) return false;
  r.pos = 4;
  if (r.u32() != 1) return false;
  p->y = r.ef();
  p->com_a_vec = r.hash();
  p->com_i = r.hash();
  p->y4 = r.ef();
  p->y5 = r.ef();
  size_t ncols = r.count(8);
  size_t nrows = r.u32();
  if (!r.ok || nrows > 1024) return false;
  p->h_cols.assign(ncols, std::vector<u64>(nrows));
  for (size_t i = 0; i < ncols && r.ok; ++i)
    for (size_t k = 0; k < nrows && r.ok; ++k) p->h_cols[i][k] = r.bf();
  p->h_open = r.bytes();
  for (SumcheckProof* s : {&p->sc_binary, &p->sc_hash, &p->sc_recon, &p->sc_table, &p->sc_rslink,
                           &p->sc_bi_batch, &p->sc_a_batch})
    *s = r.sc();
  BatchProof& b = p->batch;
  b.code_rate = r.u32();
  b.log_len = r.u32();
  size_t nch = r.count(4);
  b.reduction_msgs.assign(nch, {});
  for (size_t c = 0; c < nch && r.ok; ++c) {
    size_t k = r.count(16);
    for (size_t i = 0; i < k && r.ok; ++i) b.reduction_msgs[c].push_back(r.ef());
  }
  size_t nroots = r.count(32);
  for (size_t i = 0; i < nroots && r.ok; ++i) b.fold_roots.push_back(r.hash());
  size_t nf = r.count(16);
  for (size_t i = 0; i < nf && r.ok; ++i) b.final_codeword.push_back(r.ef());
  size_t nfo = r.count(8);
  for (size_t i = 0; i < nfo && r.ok; ++i) b.fold_openings.push_back(r.opening<EF>(16));
  size_t nbf = r.count(8);
  for (size_t i = 0; i < nbf && r.ok; ++i) b.base_bf.push_back(r.opening<u64>(8));
  size_t nef = r.count(8);
  for (size_t i = 0; i < nef && r.ok; ++i) b.base_ef.push_back(r.opening<EF>(16));
  return r.ok && r.pos == len;
}

// ---- standalone Basefold proofs ----
template <class LF>
inline std::vector<uint8_t> encode_basefold_proof(const BasefoldProof<LF>& p) {
  Writer w;
  w.b.insert(w.b.end(), {'L', 'G', 'S', 'B'});
  w.u32(1);
  w.u32(p.num_vars);
  w.u32(p.code_rate);
  w.u32(p.log_interleave);
  w.u32(std::is_same<LF, EF>::value ? 1 : 0);
  w.ef(p.claimed_eval);
  w.u32((uint32_t)p.reduction_msgs.size());
  for (auto& m : p.reduction_msgs) {
    w.ef(m.first);
    w.ef(m.second);
  }
  w.u32((uint32_t)p.fold_roots.size());
  for (auto& h : p.fold_roots) w.hash(h);
  w.u32((uint32_t)p.final_codeword.size());
  for (auto& e : p.final_codeword) w.ef(e);
  w.opening(p.base_opening);
  w.u32((uint32_t)p.fold_openings.size());
  for (auto& o : p.fold_openings) w.opening(o);
  return w.b;
}

// The leaf field of an encoded standalone Basefold proof: 0 BF, 1 EF, -1 not such a proof.
inline int basefold_proof_leaf_ef(const uint8_t* d, size_t len) {
  if (len < 24 || std::memcmp(d, "LGSB", 4) != 0) return -1;
  uint32_t v = 0;
  std::memcpy(&v, d + 20, 4);
  return v <= 1 ? (int)v : -1;
}

template <class LF>
inline bool decode_basefold_proof(const uint8_t* d, size_t len, BasefoldProof<LF>* p) {
  Reader r(d, len);
  if (!r.need(4) || std::memcmp(d, "LGSB", 4) != 0) return false;
  r.pos = 4;
  if (r.u32() != 1) return false;
  p->num_vars = r.u32();
  p->code_rate = r.u32();
  p->log_interleave = r.u32();
  if (r.u32() != (std::is_same<LF, EF>::value ? 1u : 0u)) return false;
  if (!r.ok || p->num_vars > 40 || p->code_rate > 8 || p->log_interleave > p->num_vars)
    return false;
  p->claimed_eval = r.ef();
  size_t rounds = r.count(32);
  for (size_t i = 0; i < rounds && r.ok; ++i) {
    EF a = r.ef(), b = r.ef();
    p->reduction_msgs.push_back({a, b});
  }
  size_t nroots = r.count(32);
  for (size_t i = 0; i < nroots && r.ok; ++i) p->fold_roots.push_back(r.hash());
  size_t nf = r.count(16);
  for (size_t i = 0; i < nf && r.ok; ++i) p->final_codeword.push_back(r.ef());
  p->base_opening = r.opening<LF>(sizeof(LF) == 8 ? 8 : 16);
  size_t nfo = r.count(8);
  for (size_t i = 0; i < nfo && r.ok; ++i) p->fold_openings.push_back(r.opening<EF>(16));
  return r.ok && r.pos == len;
}

}  // namespace orc
