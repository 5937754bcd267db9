// GKR fraction-sum prover (logup/src/frac_sum.rs:110-218) and the GKR-LogUp lookup prover built on
// it (logup/src/lookup.rs:119-143) on the device.
//
// The circuit is a binary tree of fraction additions over 2^k inputs: level s-1 pairs level s
// along the low bit, p' = p0 q1 + p1 q0, q' = q0 q1.  Every level is kept (level s at offset
// 2^s - 1 of the P and Q arrays); a launch of fs_build_kernel computes up to FS_BUILD_T levels of
// one subtree per CTA in shared memory.
//
// Layer r (r = 0 .. k-1) proves the claim on level r at the point z_r with a degree-3 sumcheck
// over r rounds on the low-bit splits A0, A1, B0, B1 of level r+1, binding the low bit first.
// The oracle is pre-drawn (utils/src/oracle.rs:10-64), so every layer's lambda, fold challenges
// and point are known before proving starts: the layers are independent and all run in the same
// launches.  Two identities cut the work per pair of elements and round:
//  * eq(z, .) factors: after t folds the eq vector is C_t eq(z_t, b) E_{t+1}(j), with
//    C_t = prod_{k<t} eq(z_k, c_k) a constant and E_{t+1} the eq table of z_{t+1..}.  So
//    g_t(x) = C_t l_t(x) S_t(x), l_t(x) = (1 - z_t) + x (2 z_t - 1), and S_t(x) =
//    sum_j E_{t+1}(j) H_j(x) is quadratic: S_t at 0, 1 and its leading coefficient give
//    g_t(0..3) (the host supplies K_t(x) = C_t l_t(x)).  Nothing of size 2^r is built for eq.
//  * H = A0 B1 + A1 B0 + lambda B0 B1 = A0 B1 + B0 U with U = A1 + lambda B1, and U folds like
//    A1 (folding is affine), so the stored arrays are A0, U, B0, B1: 6 products for H at 0, 1 and
//    its leading coefficient, 3 for the weights, 4 for the folds.  With all numerators one (the
//    query side of a lookup) A0 stays 1 and that drops to 3 + 3 + 3.
// A pass folds FS_B rounds: each CTA takes 2^FS_B consecutive elements of the four arrays, the
// first round straight from the level (or the previous pass's output), the rest in shared memory,
// and leaves one element per array; per-CTA sums of every round go to a scratch array that
// fs_rounds_kernel reduces into the round polynomials.  Round polynomials hold the same field
// values as the reference's (the identities are exact), so the proofs are byte-identical.
#include <algorithm>
#include <array>
#include <cstring>

#include "prover.cuh"

namespace lgs {

namespace {

constexpr unsigned FS_THREADS = 256;
constexpr unsigned FS_B = 10;        // rounds per sumcheck pass (2^FS_B elements per CTA)
constexpr unsigned FS_BUILD_T = 10;  // tree levels per build launch
constexpr unsigned FS_MAX_K = 28;

__device__ __forceinline__ ef2 ld_ef(const ef2* p) {
  const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(p);
  return ef_make(v.x, v.y);
}
__device__ __forceinline__ void st_ef(ef2* p, ef2 v) {
  *reinterpret_cast<ulonglong2*>(p) = make_ulonglong2(v.c0, v.c1);
}
__device__ __forceinline__ ef2 ef_canon(ef2 v) { return ef_make(gl_canon(v.c0), gl_canon(v.c1)); }
__device__ __forceinline__ ef2 shfl_xor_ef(ef2 v, int m) {
  return ef_make(__shfl_xor_sync(0xffffffffu, v.c0, m), __shfl_xor_sync(0xffffffffu, v.c1, m));
}

}  // namespace

// One level of the tree: a stored level, or the caller's input (numerators all one when p is
// null; denominators alpha - q[i] when q_sub is set, the lookup's alpha - a_i).
struct FsSrc {
  const ef2* p;
  const ef2* q;
  ef2 alpha;
  int q_sub;
};

namespace {

__device__ __forceinline__ ef2 src_p(const FsSrc& s, size_t i) {
  return s.p ? ef_canon(ld_ef(s.p + i)) : ef_one();
}
__device__ __forceinline__ ef2 src_q(const FsSrc& s, size_t i) {
  const ef2 v = ef_canon(ld_ef(s.q + i));
  return s.q_sub ? ef_sub(s.alpha, v) : v;
}

// Levels S-1 .. S-T of the tree from level S: CTA c reduces entries [c 2^T, (c+1) 2^T) of level
// S (frac_sum.rs:124-136).  Shared memory: a chain of the levels, p then q (2 x 2^T entries).
__global__ void __launch_bounds__(FS_THREADS)
    fs_build_kernel(FsSrc src, unsigned S, unsigned T, ef2* __restrict__ P, ef2* __restrict__ Q) {
  extern __shared__ ef2 fs_sm[];
  ef2* sp = fs_sm;
  ef2* sq = fs_sm + ((size_t)1 << T);
  const unsigned half = 1u << (T - 1);
  const size_t base = (size_t)blockIdx.x << T;
  size_t gout = (((size_t)1 << (S - 1)) - 1) + ((size_t)blockIdx.x << (T - 1));
  for (unsigned i = threadIdx.x; i < half; i += blockDim.x) {
    const size_t e = base + 2 * i;
    const ef2 q0 = src_q(src, e), q1 = src_q(src, e + 1);
    ef2 np;
    if (src.p)
      np = ef_add(ef_mul(src_p(src, e), q1), ef_mul(src_p(src, e + 1), q0));
    else
      np = ef_add(q1, q0);  // 1 q1 + 1 q0
    const ef2 nq = ef_mul(q0, q1);
    sp[i] = np;
    sq[i] = nq;
    st_ef(P + gout + i, np);
    st_ef(Q + gout + i, nq);
  }
  unsigned off = 0, cnt = half;
  for (unsigned l = 2; l <= T; ++l) {
    __syncthreads();
    const unsigned nc = cnt >> 1;
    gout = (((size_t)1 << (S - l)) - 1) + ((size_t)blockIdx.x << (T - l));
    for (unsigned i = threadIdx.x; i < nc; i += blockDim.x) {
      const ef2 p0 = sp[off + 2 * i], p1 = sp[off + 2 * i + 1];
      const ef2 q0 = sq[off + 2 * i], q1 = sq[off + 2 * i + 1];
      const ef2 np = ef_add(ef_mul(p0, q1), ef_mul(p1, q0)), nq = ef_mul(q0, q1);
      sp[off + cnt + i] = np;
      sq[off + cnt + i] = nq;
      st_ef(P + gout + i, np);
      st_ef(Q + gout + i, nq);
    }
    off += cnt;
    cnt = nc;
  }
}

}  // namespace

// One pass of one layer: rounds t0 .. t0+nb-1 of the layer-r sumcheck.
struct FsJob {
  FsSrc src;          // the first pass reads level r+1 (entries 2i, 2i+1 are element i)
  const ef2* fin;     // later passes: the previous pass's arrays A0 | U | B0 | B1 (n each)
  ef2* fout;          // this pass's arrays (ncta each); on the layer's last pass, the leaves
  ef2* part;          // per-round, per-CTA sums: [tau][cta][S(0), S(1), leading coefficient]
  const ef2* z;       // the layer's point z_r (r coordinates)
  const ef2* ch;      // the layer's fold challenges (r)
  ef2 lambda;
  size_t n;           // elements per array at round t0 (2^(r - t0))
  unsigned r, t0, nb, ncta, first_cta;
  int ones;           // A0 == 1 throughout (numerators all one)
};

// Reduction of one round: the CTA sums of the pass that ran it, times K_t(0..3).
struct FsRound {
  const ef2* part;  // ncta x 3
  ef2* out;         // g(0), g(1), g(2), g(3)
  ef2 K[4];
  unsigned ncta;
};

namespace {

struct Q4 {
  ef2 a0, u, b0, b1;
};

// One pair (lo = element 2j, hi = element 2j+1) of round t: adds w H(0), w H(1) and w times the
// leading coefficient of H to s, and returns the element folded with c.
__device__ __forceinline__ Q4 fs_pair(const Q4& lo, const Q4& hi, ef2 w, ef2 c, bool ones,
                                      ef2 (&s)[3]) {
  const ef2 du = ef_sub(hi.u, lo.u), db0 = ef_sub(hi.b0, lo.b0), db1 = ef_sub(hi.b1, lo.b1);
  ef2 h0, h1, h2;
  Q4 o;
  if (ones) {
    h0 = ef_add(lo.b1, ef_mul(lo.b0, lo.u));
    h1 = ef_add(hi.b1, ef_mul(hi.b0, hi.u));
    h2 = ef_mul(db0, du);
    o.a0 = ef_one();
  } else {
    const ef2 da0 = ef_sub(hi.a0, lo.a0);
    h0 = ef_add(ef_mul(lo.a0, lo.b1), ef_mul(lo.b0, lo.u));
    h1 = ef_add(ef_mul(hi.a0, hi.b1), ef_mul(hi.b0, hi.u));
    h2 = ef_add(ef_mul(da0, db1), ef_mul(db0, du));
    o.a0 = ef_add(lo.a0, ef_mul(c, da0));
  }
  s[0] = ef_add(s[0], ef_mul(w, h0));
  s[1] = ef_add(s[1], ef_mul(w, h1));
  s[2] = ef_add(s[2], ef_mul(w, h2));
  o.u = ef_add(lo.u, ef_mul(c, du));
  o.b0 = ef_add(lo.b0, ef_mul(c, db0));
  o.b1 = ef_add(lo.b1, ef_mul(c, db1));
  return o;
}

__device__ __forceinline__ Q4 job_load(const FsJob& jb, size_t e) {
  Q4 x;
  if (jb.fin) {
    x.a0 = ld_ef(jb.fin + e);
    x.u = ld_ef(jb.fin + jb.n + e);
    x.b0 = ld_ef(jb.fin + 2 * jb.n + e);
    x.b1 = ld_ef(jb.fin + 3 * jb.n + e);
  } else {
    x.b0 = src_q(jb.src, 2 * e);
    x.b1 = src_q(jb.src, 2 * e + 1);
    if (jb.ones) {
      x.a0 = ef_one();
      x.u = ef_add(ef_one(), ef_mul(jb.lambda, x.b1));
    } else {
      x.a0 = src_p(jb.src, 2 * e);
      x.u = ef_add(src_p(jb.src, 2 * e + 1), ef_mul(jb.lambda, x.b1));
    }
  }
  return x;
}

__device__ __forceinline__ void warp_sum3(ef2 (&s)[3]) {
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int m = 16; m; m >>= 1) s[q] = ef_add(s[q], shfl_xor_ef(s[q], m));
}

// Sum s over the CTA and store it at dst (3 EF).  Every thread must call it.
__device__ void block_store3(ef2 (&s)[3], ef2* red, ef2* dst) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  warp_sum3(s);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 3; ++q) red[q * 32 + warp] = s[q];
  __syncthreads();
  if (warp == 0) {
    ef2 v[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) v[q] = lane < nw ? red[q * 32 + lane] : ef_zero();
    warp_sum3(v);
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < 3; ++q) st_ef(dst + q, v[q]);
  }
  __syncthreads();
}

// Shared memory of a pass: the weight tables (2^FS_B entries), the folded elements after the
// first round (2^(FS_B-1) x 4) and the reduction scratch (3 x 32).
constexpr size_t FS_PASS_SMEM =
    ((size_t)1 << FS_B) * sizeof(ef2) + ((size_t)1 << (FS_B - 1)) * sizeof(Q4) + 96 * sizeof(ef2);

__global__ void __launch_bounds__(FS_THREADS)
    fs_pass_kernel(const FsJob* __restrict__ jobs, unsigned njobs) {
  extern __shared__ ef2 fs_sm[];
  ef2* wt = fs_sm;                                     // W_tau at offset 2^(nb - tau - 1) - 1
  Q4* xs = reinterpret_cast<Q4*>(fs_sm + (1u << FS_B));
  ef2* red = fs_sm + (1u << FS_B) + 4 * (1u << (FS_B - 1));
  unsigned ji = 0;
  while (ji + 1 < njobs && blockIdx.x >= jobs[ji + 1].first_cta) ++ji;
  const FsJob& jb = jobs[ji];
  const unsigned cta = blockIdx.x - jb.first_cta, nb = jb.nb, t0 = jb.t0, r = jb.r;
  const bool ones = jb.ones != 0;

  // W_{nb-1} = [prod over k in [t0+nb, r) of eq(z_k, bit k-t0-nb of cta)]; then
  // W_tau[2m + b] = W_{tau+1}[m] eq(z_{t0+tau+1}, b): the weight of local pair jl in round
  // t0+tau is W_tau[jl] = E_{t+1}(cta 2^(nb-tau-1) + jl).
  if (threadIdx.x < 32) {
    ef2 f = ef_one();
    const unsigned k = t0 + nb + threadIdx.x;
    if (k < r) {
      const ef2 zk = ld_ef(jb.z + k);
      f = ((cta >> threadIdx.x) & 1) ? zk : ef_sub(ef_one(), zk);
    }
#pragma unroll
    for (int m = 16; m; m >>= 1) f = ef_mul(f, shfl_xor_ef(f, m));
    if (threadIdx.x == 0) wt[0] = f;
  }
  for (int tau = (int)nb - 2; tau >= 0; --tau) {
    __syncthreads();
    const unsigned sz = 1u << (nb - tau - 1), prev = (sz >> 1) - 1, off = sz - 1;
    const ef2 z1 = ld_ef(jb.z + t0 + tau + 1), z0 = ef_sub(ef_one(), z1);
    for (unsigned i = threadIdx.x; i < sz; i += blockDim.x)
      wt[off + i] = ef_mul(wt[prev + (i >> 1)], (i & 1) ? z1 : z0);
  }
  __syncthreads();

  // round t0: straight from global memory
  {
    const unsigned np = 1u << (nb - 1);
    const ef2 c = ld_ef(jb.ch + t0);
    ef2 s[3] = {ef_zero(), ef_zero(), ef_zero()};
    for (unsigned jl = threadIdx.x; jl < np; jl += blockDim.x) {
      const size_t e = ((size_t)cta << nb) + 2 * jl;
      const Q4 lo = job_load(jb, e), hi = job_load(jb, e + 1);
      xs[jl] = fs_pair(lo, hi, wt[np - 1 + jl], c, ones, s);
    }
    block_store3(s, red, jb.part + (size_t)cta * 3);
  }
  // rounds t0+1 .. t0+nb-1 in shared memory (at most 2^(FS_B-2) = blockDim pairs)
  for (unsigned tau = 1; tau < nb; ++tau) {
    const unsigned np = 1u << (nb - tau - 1);
    const ef2 c = ld_ef(jb.ch + t0 + tau);
    ef2 s[3] = {ef_zero(), ef_zero(), ef_zero()};
    Q4 o;
    const bool act = threadIdx.x < np;
    if (act) o = fs_pair(xs[2 * threadIdx.x], xs[2 * threadIdx.x + 1], wt[np - 1 + threadIdx.x], c,
                         ones, s);
    __syncthreads();
    if (act) xs[threadIdx.x] = o;
    block_store3(s, red, jb.part + ((size_t)tau * jb.ncta + cta) * 3);
  }
  if (threadIdx.x == 0) {
    const Q4 x = xs[0];
    st_ef(jb.fout + cta, x.a0);
    st_ef(jb.fout + jb.ncta + cta, x.u);
    st_ef(jb.fout + 2 * jb.ncta + cta, x.b0);
    st_ef(jb.fout + 3 * jb.ncta + cta, x.b1);
  }
}

// g(x) = K(x) S(x) with S quadratic: S(2) = -S(0) + 2 S(1) + 2 L, S(3) = -2 S(0) + 3 S(1) + 6 L
// (L the leading coefficient).
__global__ void __launch_bounds__(FS_THREADS) fs_rounds_kernel(const FsRound* __restrict__ rounds) {
  __shared__ ef2 red[96];
  const FsRound& rd = rounds[blockIdx.x];
  ef2 s[3] = {ef_zero(), ef_zero(), ef_zero()};
  for (unsigned i = threadIdx.x; i < rd.ncta; i += blockDim.x)
#pragma unroll
    for (int q = 0; q < 3; ++q) s[q] = ef_add(s[q], ld_ef(rd.part + (size_t)i * 3 + q));
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  warp_sum3(s);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 3; ++q) red[q * 32 + warp] = s[q];
  __syncthreads();
  if (warp != 0) return;
#pragma unroll
  for (int q = 0; q < 3; ++q) s[q] = lane < nw ? red[q * 32 + lane] : ef_zero();
  warp_sum3(s);
  if (lane != 0) return;
  const ef2 s0 = s[0], s1 = s[1], l = s[2];
  const ef2 two_s1 = ef_add(s1, s1), two_l = ef_add(l, l);
  const ef2 s2 = ef_sub(ef_add(two_s1, two_l), s0);
  const ef2 s3 = ef_sub(ef_add(ef_add(two_s1, s1), ef_add(ef_add(two_l, two_l), two_l)),
                        ef_add(s0, s0));
  st_ef(rd.out + 0, ef_mul(rd.K[0], s0));
  st_ef(rd.out + 1, ef_mul(rd.K[1], s1));
  st_ef(rd.out + 2, ef_mul(rd.K[2], s2));
  st_ef(rd.out + 3, ef_mul(rd.K[3], s3));
}

// num, den (level 0) and level 1's four entries (layer 0's leaves).
__global__ void fs_root_kernel(FsSrc l1, const ef2* P, const ef2* Q, ef2* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st_ef(out + 0, ld_ef(P));
  st_ef(out + 1, ld_ef(Q));
  st_ef(out + 2, src_p(l1, 0));
  st_ef(out + 3, src_p(l1, 1));
  st_ef(out + 4, src_q(l1, 0));
  st_ef(out + 5, src_q(l1, 1));
}
// k == 0: the single fraction is the root and the reduced claim.
__global__ void fs_single_kernel(FsSrc in, ef2* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st_ef(out + 0, src_p(in, 0));
  st_ef(out + 1, src_q(in, 0));
}

// Host field helpers (challenge bookkeeping).
ef2 h_eq1(const ef2& z, const ef2& c) {  // z c + (1 - z)(1 - c)
  return ef_add(ef_mul(z, c), ef_mul(ef_sub(ef_one(), z), ef_sub(ef_one(), c)));
}

size_t ceil256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

// The device plan of one fraction-sum proof: what fs_enqueue launched, what the host reads back.
struct FsPlan {
  unsigned k = 0;
  uint64_t f0 = 0;              // fields cursor at the start
  std::vector<ef2> lambda, beta;
  std::vector<std::vector<ef2>> z, ch;
  size_t stage_off = 0;         // EF offset of this proof's values in the staging area
  size_t round_off = 0;         // EF offset of the round polynomials (within the staging)
  size_t stage_elems = 0;
};

static size_t fs_fields_needed(unsigned k) { return (size_t)k * (k + 3) / 2; }

// Enqueues one fraction-sum proof of 2^k inputs on st.  Its values land in `stage` (device) at
// plan->stage_off: num, den, level-1 entries (6 EF), then per layer r >= 1 the leaves
// (A0, U, B0, B1), then the round polynomials layer by layer.
static void fs_enqueue(lgs_ctx* c, const FsSrc& in, unsigned k, const u64* fields, size_t nfields,
                       uint64_t f0, ef2* stage, size_t stage_off, FsPlan* plan, cudaStream_t st) {
  Arena& ar = c->arena;
  if (k > FS_MAX_K) throw ShapeError("frac_sum: at most 2^28 fractions");
  const size_t need = fs_fields_needed(k);
  if (f0 > nfields || nfields - f0 < need) throw OracleError("oracle exhausted (fields)");
  plan->k = k;
  plan->f0 = f0;
  plan->stage_off = stage_off;
  auto F = [&](size_t i) { return ef_make(gl_canon(fields[2 * (f0 + i)]), gl_canon(fields[2 * (f0 + i) + 1])); };
  plan->lambda.assign(k, ef_zero());
  plan->beta.assign(k, ef_zero());
  plan->z.assign(k, {});
  plan->ch.assign(k, {});
  for (unsigned r = 0; r < k; ++r) {  // frac_sum.rs:143-160: lambda, r fold challenges, beta
    const size_t o = (size_t)r * (r + 3) / 2;
    plan->lambda[r] = F(o);
    for (unsigned t = 0; t < r; ++t) plan->ch[r].push_back(F(o + 1 + t));
    plan->beta[r] = F(o + 1 + r);
    if (r > 0) {
      plan->z[r].push_back(plan->beta[r - 1]);
      plan->z[r].insert(plan->z[r].end(), plan->ch[r - 1].begin(), plan->ch[r - 1].end());
    }
  }
  size_t nrounds = 0;
  for (unsigned r = 1; r < k; ++r) nrounds += r;
  plan->round_off = stage_off + 6 + 4 * (k ? k - 1 : 0);
  plan->stage_elems = 6 + 4 * (k ? k - 1 : 0) + 4 * nrounds;
  if (k == 0) {
    fs_single_kernel<<<1, 32, 0, st>>>(in, stage + stage_off);
    LGS_LAUNCH_CHECK();
    plan->stage_elems = 2;
    return;
  }

  // ---- levels ---------------------------------------------------------------------------
  const size_t nlev = ((size_t)1 << k) - 1;  // levels 0 .. k-1
  ef2* P = ar.get<ef2>(nlev);
  ef2* Q = ar.get<ef2>(nlev);
  {
    unsigned S = k;
    FsSrc src = in;
    while (S > 0) {
      const unsigned T = std::min(S, FS_BUILD_T);
      const size_t smem = 2 * ((size_t)1 << T) * sizeof(ef2);
      fs_build_kernel<<<(unsigned)((size_t)1 << (S - T)), FS_THREADS, smem, st>>>(src, S, T, P, Q);
      LGS_LAUNCH_CHECK();
      S -= T;
      src = FsSrc{P + ((size_t)1 << S) - 1, Q + ((size_t)1 << S) - 1, ef_zero(), 0};
    }
  }
  auto level = [&](unsigned s) -> FsSrc {
    if (s == k) return in;
    return FsSrc{P + ((size_t)1 << s) - 1, Q + ((size_t)1 << s) - 1, ef_zero(), 0};
  };

  // ---- parameter blob: per layer z and challenges; jobs per pass; rounds ------------------
  const unsigned npass = k > 1 ? (k - 2) / FS_B + 1 : 0;  // layer k-1 has k-1 rounds
  std::vector<std::vector<FsJob>> jobs(npass);
  std::vector<FsRound> rounds;
  std::vector<ef2> zc;  // z_r then ch_r for every layer r >= 1
  std::vector<size_t> zoff(k, 0);
  for (unsigned r = 1; r < k; ++r) {
    zoff[r] = zc.size();
    zc.insert(zc.end(), plan->z[r].begin(), plan->z[r].end());
    zc.insert(zc.end(), plan->ch[r].begin(), plan->ch[r].end());
  }
  size_t up_bytes = ceil256(zc.size() * sizeof(ef2));
  const size_t up_jobs = up_bytes;
  size_t total_jobs = 0;
  for (unsigned r = 1; r < k; ++r) total_jobs += (r - 1) / FS_B + 1;
  up_bytes += ceil256(total_jobs * sizeof(FsJob));
  const size_t up_rounds = up_bytes;
  up_bytes += ceil256(nrounds * sizeof(FsRound));
  uint8_t* d_up = ar.get<uint8_t>(up_bytes);
  std::vector<uint8_t> h_up(up_bytes, 0);
  std::memcpy(h_up.data(), zc.data(), zc.size() * sizeof(ef2));
  const ef2* d_zc = (const ef2*)d_up;

  size_t round_pos = plan->round_off;
  for (unsigned r = 1; r < k; ++r) {
    const ef2* z = d_zc + zoff[r];
    const ef2* chp = z + r;
    // C_t = prod_{s<t} eq(z_s, c_s); K_t(x) = C_t ((1 - z_t) + x (2 z_t - 1))
    ef2 C = ef_one();
    std::vector<std::array<ef2, 4>> K(r);
    for (unsigned t = 0; t < r; ++t) {
      const ef2 zt = plan->z[r][t];
      const ef2 l0 = ef_sub(ef_one(), zt), d = ef_sub(ef_add(zt, zt), ef_one());
      ef2 l = l0;
      for (int x = 0; x < 4; ++x) {
        K[t][x] = ef_mul(C, l);
        l = ef_add(l, d);
      }
      C = ef_mul(C, h_eq1(zt, plan->ch[r][t]));
    }
    const ef2* fin = nullptr;
    for (unsigned t0 = 0, pi = 0; t0 < r; t0 += FS_B, ++pi) {
      const unsigned nb = std::min(FS_B, r - t0);
      FsJob jb{};
      jb.src = level(r + 1);
      jb.fin = fin;
      jb.n = (size_t)1 << (r - t0);
      jb.ncta = 1u << (r - t0 - nb);
      jb.fout = t0 + nb == r ? stage + stage_off + 6 + 4 * (r - 1) : ar.get<ef2>(4 * (size_t)jb.ncta);
      jb.part = ar.get<ef2>((size_t)nb * jb.ncta * 3);
      jb.z = z;
      jb.ch = chp;
      jb.lambda = plan->lambda[r];
      jb.r = r;
      jb.t0 = t0;
      jb.nb = nb;
      jb.ones = (r + 1 == k && in.p == nullptr) ? 1 : 0;
      jobs[pi].push_back(jb);
      for (unsigned tau = 0; tau < nb; ++tau) {
        FsRound rd{};
        rd.part = jb.part + (size_t)tau * jb.ncta * 3;
        rd.out = stage + round_pos + 4 * (t0 + tau);
        for (int x = 0; x < 4; ++x) rd.K[x] = K[t0 + tau][x];
        rd.ncta = jb.ncta;
        rounds.push_back(rd);
      }
      fin = jb.fout;
    }
    round_pos += 4 * (size_t)r;
  }
  {
    size_t o = up_jobs;
    for (auto& pj : jobs) {
      unsigned first = 0;
      for (auto& jb : pj) {
        jb.first_cta = first;
        first += jb.ncta;
      }
      std::memcpy(h_up.data() + o, pj.data(), pj.size() * sizeof(FsJob));
      o += pj.size() * sizeof(FsJob);
    }
    std::memcpy(h_up.data() + up_rounds, rounds.data(), rounds.size() * sizeof(FsRound));
  }
  LGS_CUDA(cudaMemcpyAsync(d_up, h_up.data(), up_bytes, cudaMemcpyHostToDevice, st));
  // the blob is pageable host memory: the copy is complete (staged) when the call returns

  // ---- passes, rounds, root --------------------------------------------------------------
  static bool attr_set = false;
  if (!attr_set) {
    LGS_CUDA(cudaFuncSetAttribute(fs_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)FS_PASS_SMEM));
    attr_set = true;
  }
  {
    const FsJob* dj = (const FsJob*)(d_up + up_jobs);
    for (auto& pj : jobs) {
      unsigned ctas = 0;
      for (auto& jb : pj) ctas += jb.ncta;
      fs_pass_kernel<<<ctas, FS_THREADS, FS_PASS_SMEM, st>>>(dj, (unsigned)pj.size());
      LGS_LAUNCH_CHECK();
      dj += pj.size();
    }
  }
  if (!rounds.empty()) {
    fs_rounds_kernel<<<(unsigned)rounds.size(), FS_THREADS, 0, st>>>(
        (const FsRound*)(d_up + up_rounds));
    LGS_LAUNCH_CHECK();
  }
  fs_root_kernel<<<1, 32, 0, st>>>(level(1), P, Q, stage + stage_off);
  LGS_LAUNCH_CHECK();
}

// Assembles the "LGSF" encoding of one proof from the staged values and returns the reduced
// claim (frac_sum.rs:143-160).
static void fs_assemble(const FsPlan& pl, const ef2* hst, ByteWriter& w, std::vector<ef2>* point,
                        ef2* pe, ef2* qe) {
  const unsigned k = pl.k;
  w.u32v(0x4653474Cu);  // "LGSF"
  w.u32v(1);
  const ef2* v = hst + pl.stage_off;
  auto ef = [&](const ef2& e) {
    w.bf(e.c0);
    w.bf(e.c1);
  };
  ef(v[0]);
  ef(v[1]);
  w.u32v(k);
  point->clear();
  if (k == 0) {
    *pe = v[0];
    *qe = v[1];
    return;
  }
  std::array<ef2, 4> leaves{};
  for (unsigned r = 0; r < k; ++r) {
    w.u32v(r);
    if (r == 0) {
      leaves = {v[2], v[3], v[4], v[5]};
    } else {
      const ef2* rp = hst + pl.round_off;
      size_t off = 0;
      for (unsigned s = 1; s < r; ++s) off += 4 * (size_t)s;
      w.bf_run(&rp[off].c0, 8 * (size_t)r);
      const ef2* lv = v + 6 + 4 * (r - 1);
      // A1 = U - lambda B1
      leaves = {lv[0], ef_sub(lv[1], ef_mul(pl.lambda[r], lv[3])), lv[2], lv[3]};
    }
    for (const ef2& e : leaves) ef(e);
  }
  const ef2 beta = pl.beta[k - 1];
  point->push_back(beta);
  point->insert(point->end(), pl.ch[k - 1].begin(), pl.ch[k - 1].end());
  *pe = ef_add(ef_mul(ef_sub(ef_one(), beta), leaves[0]), ef_mul(beta, leaves[1]));
  *qe = ef_add(ef_mul(ef_sub(ef_one(), beta), leaves[2]), ef_mul(beta, leaves[3]));
}

static unsigned log2_exact(size_t n, const char* what) {
  if (n == 0 || (n & (n - 1))) throw ShapeError(std::string(what) + ": a power-of-two length");
  unsigned k = 0;
  while (((size_t)1 << k) < n) ++k;
  return k;
}

// Device copy of n EF values (host or device source), canonical values left to the kernels.
static const ef2* fs_input(lgs_ctx* c, const u64* src, size_t n, bool on_device, cudaStream_t st) {
  if (!src) return nullptr;
  if (on_device) {
    if (((uintptr_t)src & 15) != 0) throw ShapeError("frac_sum: device input must be 16-byte aligned");
    return (const ef2*)src;
  }
  ef2* d = c->arena.get<ef2>(n);
  h2d_staged(c, d, src, n * sizeof(ef2), st);
  return d;
}

void frac_sum_prove_dev(lgs_ctx* c, const u64* p, const u64* q, size_t n, bool on_device,
                        const u64* fields, size_t nfields, uint64_t* cursor,
                        std::vector<uint8_t>* proof_out, u64* point_out, u64* claim_out) {
  const unsigned k = log2_exact(n, "frac_sum");
  if (!q) throw ShapeError("frac_sum: denominators required");
  cudaStream_t st = c->st;
  c->arena.begin();
  FsSrc in{fs_input(c, p, n, on_device, st), fs_input(c, q, n, on_device, st), ef_zero(), 0};
  size_t nrounds = 0;
  for (unsigned r = 1; r < k; ++r) nrounds += r;
  const size_t elems = 6 + 4 * (size_t)k + 4 * nrounds;
  ef2* stage = c->arena.get<ef2>(elems);
  FsPlan pl;
  fs_enqueue(c, in, k, fields, nfields, *cursor, stage, 0, &pl, st);
  c->down.reserve(elems * sizeof(ef2));
  ef2* hst = c->down.as<ef2>();
  LGS_CUDA(cudaMemcpyAsync(hst, stage, pl.stage_elems * sizeof(ef2), cudaMemcpyDeviceToHost, st));
  LGS_CUDA(cudaStreamSynchronize(st));
  ByteWriter w(*proof_out);
  std::vector<ef2> pt;
  ef2 pe, qe;
  fs_assemble(pl, hst, w, &pt, &pe, &qe);
  w.finish_in_place();
  for (size_t i = 0; i < pt.size(); ++i) {
    point_out[2 * i] = pt[i].c0;
    point_out[2 * i + 1] = pt[i].c1;
  }
  claim_out[0] = pe.c0;
  claim_out[1] = pe.c1;
  claim_out[2] = qe.c0;
  claim_out[3] = qe.c1;
  *cursor += fs_fields_needed(k);
}

// lookup::prove_with_opening_points: alpha, the query circuit (numerators one, denominators
// alpha - a_i) and the table circuit (numerators e_j, denominators alpha - t_j).  The table side
// runs on a side stream beside the query side.
void lookup_prove_dev(lgs_ctx* c, const u64* a, size_t m, const u64* t, const u64* e, size_t n,
                      bool on_device, const u64* fields, size_t nfields, uint64_t* cursor,
                      std::vector<uint8_t>* proof_out, u64* zq_out, u64* zt_out) {
  const unsigned kq = log2_exact(m, "lookup queries"), kt = log2_exact(n, "lookup table");
  if (!a || !t || !e) throw ShapeError("lookup: a, t and e are required");
  const uint64_t f0 = *cursor;
  if (f0 >= nfields) throw OracleError("oracle exhausted (fields)");
  const ef2 alpha = ef_make(gl_canon(fields[2 * f0]), gl_canon(fields[2 * f0 + 1]));
  cudaStream_t st = c->st, sd = c->side[0];
  c->arena.begin();
  size_t rq = 0, rt = 0;
  for (unsigned r = 1; r < kq; ++r) rq += r;
  for (unsigned r = 1; r < kt; ++r) rt += r;
  const size_t eq_n = 6 + 4 * (size_t)kq + 4 * rq, et_n = 6 + 4 * (size_t)kt + 4 * rt;
  ef2* stage = c->arena.get<ef2>(eq_n + et_n);
  const ef2* da = fs_input(c, a, m, on_device, st);
  const ef2* dt = fs_input(c, t, n, on_device, st);
  const ef2* de = fs_input(c, e, n, on_device, st);
  LGS_CUDA(cudaEventRecord(c->ev_fork, st));
  LGS_CUDA(cudaStreamWaitEvent(sd, c->ev_fork, 0));
  FsPlan pq, ptab;
  fs_enqueue(c, FsSrc{nullptr, da, alpha, 1}, kq, fields, nfields, f0 + 1, stage, 0, &pq, st);
  fs_enqueue(c, FsSrc{de, dt, alpha, 1}, kt, fields, nfields, f0 + 1 + fs_fields_needed(kq), stage,
             eq_n, &ptab, sd);
  LGS_CUDA(cudaEventRecord(c->ev_done[0], sd));
  LGS_CUDA(cudaStreamWaitEvent(st, c->ev_done[0], 0));
  c->down.reserve((eq_n + et_n) * sizeof(ef2));
  ef2* hst = c->down.as<ef2>();
  LGS_CUDA(cudaMemcpyAsync(hst, stage, (eq_n + et_n) * sizeof(ef2), cudaMemcpyDeviceToHost, st));
  LGS_CUDA(cudaStreamSynchronize(st));
  ByteWriter w(*proof_out);
  w.u32v(0x4C53474Cu);  // "LGSL"
  w.u32v(1);
  std::vector<ef2> zq, zt;
  ef2 pe, qe;
  fs_assemble(pq, hst, w, &zq, &pe, &qe);
  fs_assemble(ptab, hst, w, &zt, &pe, &qe);
  w.finish_in_place();
  for (size_t i = 0; i < zq.size(); ++i) {
    zq_out[2 * i] = zq[i].c0;
    zq_out[2 * i + 1] = zq[i].c1;
  }
  for (size_t i = 0; i < zt.size(); ++i) {
    zt_out[2 * i] = zt[i].c0;
    zt_out[2 * i + 1] = zt[i].c1;
  }
  *cursor = f0 + 1 + fs_fields_needed(kq) + fs_fields_needed(kt);
}

}  // namespace lgs
