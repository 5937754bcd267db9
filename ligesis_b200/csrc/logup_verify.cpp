// Host verifiers of the GKR fraction sum (logup/src/frac_sum.rs:221-258) and the GKR-LogUp lookup
// (logup/src/lookup.rs:191-229) over the "LGSF" / "LGSL" encodings frac_sum.cu writes.  Cheap CPU
// work (k layers of at most k rounds), run on the caller's thread like the reference's verifier.
#include <array>
#include <vector>

#include "prover.cuh"

namespace lgs {

namespace {

struct FsLayerH {
  std::vector<std::array<ef2, 4>> polys;
  std::array<ef2, 4> leaves;
};
struct FsProofH {
  ef2 num, den;
  std::vector<FsLayerH> layers;
};

bool decode_fs(ByteReader& r, FsProofH* pf) {
  if (r.u32v() != 0x4653474Cu || r.u32v() != 1) return false;
  pf->num = r.ef();
  pf->den = r.ef();
  const uint32_t nl = r.u32v();
  if (!r.ok || nl > 64) return false;
  pf->layers.resize(nl);
  for (auto& L : pf->layers) {
    const uint32_t nr = r.u32v();
    if (!r.ok || nr > 64) return false;
    L.polys.resize(nr);
    for (auto& g : L.polys)
      for (ef2& v : g) v = r.ef();
    for (ef2& v : L.leaves) v = r.ef();
    if (!r.ok) return false;
  }
  return r.ok;
}

struct Fields {
  const u64* f;
  size_t nf;
  uint64_t cur;
  ef2 next() {
    if (cur >= nf) throw OracleError("oracle exhausted (fields)");
    const ef2 v = ef_make(gl_canon(f[2 * cur]), gl_canon(f[2 * cur + 1]));
    ++cur;
    return v;
  }
};

// interp4 (frac_sum.rs:88-106): Lagrange through (0..3, ev) at x; denominators -6, 2, -2, 6.
ef2 interp4(const std::array<ef2, 4>& ev, const ef2& x) {
  const ef2 one = ef_one(), two = ef_add(one, one), three = ef_add(two, one);
  const ef2 six = ef_mul(two, three);
  const ef2 nodes[4] = {ef_zero(), one, two, three};
  const ef2 den[4] = {ef_sub(ef_zero(), six), two, ef_sub(ef_zero(), two), six};
  ef2 acc = ef_zero();
  for (int k = 0; k < 4; ++k) {
    ef2 num = one;
    for (int m = 0; m < 4; ++m)
      if (m != k) num = ef_mul(num, ef_sub(x, nodes[m]));
    acc = ef_add(acc, ef_mul(ef_mul(ev[k], num), ef_inv(den[k])));
  }
  return acc;
}

ef2 eq_eval(const std::vector<ef2>& z, const std::vector<ef2>& zp) {
  ef2 acc = ef_one();
  for (size_t i = 0; i < z.size() && i < zp.size(); ++i)
    acc = ef_mul(acc, ef_add(ef_mul(z[i], zp[i]),
                             ef_mul(ef_sub(ef_one(), z[i]), ef_sub(ef_one(), zp[i]))));
  return acc;
}

// frac_sum::verify; false where the reference returns None.
bool fs_verify(const FsProofH& pf, Fields& o, std::vector<ef2>* point, ef2* pe, ef2* qe) {
  std::vector<ef2> z;
  ef2 p_cur = pf.num, q_cur = pf.den;
  for (size_t r = 0; r < pf.layers.size(); ++r) {
    const ef2 lambda = o.next();
    const FsLayerH& L = pf.layers[r];
    if (L.polys.size() != r) return false;
    ef2 cur = ef_add(p_cur, ef_mul(lambda, q_cur));
    std::vector<ef2> zp;
    for (const auto& g : L.polys) {
      if (!ef_eq(ef_add(g[0], g[1]), cur)) return false;
      const ef2 c = o.next();
      cur = interp4(g, c);
      zp.push_back(c);
    }
    const ef2 a0 = L.leaves[0], a1 = L.leaves[1], b0 = L.leaves[2], b1 = L.leaves[3];
    const ef2 h = ef_add(ef_add(ef_mul(a0, b1), ef_mul(a1, b0)), ef_mul(ef_mul(lambda, b0), b1));
    if (!ef_eq(cur, ef_mul(eq_eval(z, zp), h))) return false;
    const ef2 beta = o.next();
    z.clear();
    z.push_back(beta);
    z.insert(z.end(), zp.begin(), zp.end());
    const ef2 nb = ef_sub(ef_one(), beta);
    p_cur = ef_add(ef_mul(nb, a0), ef_mul(beta, a1));
    q_cur = ef_add(ef_mul(nb, b0), ef_mul(beta, b1));
  }
  *point = z;
  *pe = p_cur;
  *qe = q_cur;
  return true;
}

void put(const std::vector<ef2>& v, u64* out) {
  for (size_t i = 0; i < v.size(); ++i) {
    out[2 * i] = v[i].c0;
    out[2 * i + 1] = v[i].c1;
  }
}
void put1(const ef2& v, u64* out) {
  out[0] = v.c0;
  out[1] = v.c1;
}

}  // namespace

int frac_sum_verify_host(const uint8_t* proof, size_t len, const u64* fields, size_t nfields,
                         uint64_t* cursor, u64* point, size_t point_cap, u64* claim) {
  ByteReader r(proof, len);
  FsProofH pf;
  if (!decode_fs(r, &pf) || r.pos != len || pf.layers.size() > point_cap) return 0;
  Fields o{fields, nfields, *cursor};
  std::vector<ef2> pt;
  ef2 pe, qe;
  bool ok;
  try {
    ok = fs_verify(pf, o, &pt, &pe, &qe);
  } catch (const OracleError&) {
    ok = false;
  }
  *cursor = o.cur;
  if (!ok) return 0;
  put(pt, point);
  put1(pe, claim);
  put1(qe, claim + 2);
  return 1;
}

int lookup_verify_host(const uint8_t* proof, size_t len, const u64* fields, size_t nfields,
                       uint64_t* cursor, u64* zq, size_t zq_cap, u64* zt, size_t zt_cap,
                       u64* vals) {
  ByteReader r(proof, len);
  FsProofH q, t;
  if (r.u32v() != 0x4C53474Cu || r.u32v() != 1 || !decode_fs(r, &q) || !decode_fs(r, &t) ||
      r.pos != len || q.layers.size() > zq_cap || t.layers.size() > zt_cap)
    return 0;
  Fields o{fields, nfields, *cursor};
  bool ok = false;
  std::vector<ef2> pq, pt;
  ef2 pq_in, qq_in, pt_in, qt_in, alpha;
  try {
    alpha = o.next();
    ok = fs_verify(q, o, &pq, &pq_in, &qq_in) && fs_verify(t, o, &pt, &pt_in, &qt_in);
  } catch (const OracleError&) {
    ok = false;
  }
  *cursor = o.cur;
  if (!ok) return 0;
  if (!ef_eq(pq_in, ef_one())) return 0;  // the query numerator is the constant one
  if (!ef_eq(ef_mul(q.num, t.den), ef_mul(t.num, q.den))) return 0;
  put(pq, zq);
  put(pt, zt);
  put1(ef_sub(alpha, qq_in), vals);  // a(zq) = alpha - qq_in
  put1(pt_in, vals + 2);             // e(zt)
  put1(ef_sub(alpha, qt_in), vals + 4);  // t(zt) = alpha - qt_in
  return 1;
}

}  // namespace lgs
