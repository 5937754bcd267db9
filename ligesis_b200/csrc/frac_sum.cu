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
//    A1 (folding is affine), so the stored arrays are A0, U, B0, B1.
//  * S_t(1) follows from the claim: (1 - z_t) S_t(0) + z_t S_t(1) = sigma_t, with sigma_0 the
//    layer's claim and sigma_{t+1} = S_t(c_t).  So a pair costs 4 products for H at 0 and its
//    leading coefficient, 2 for the weights and 4 for the folds; with all numerators one (the
//    query side of a lookup) A0 stays 1: 2 + 2 + 3.  A layer with a zero coordinate in its point
//    sums S(1) as well.
// While a layer's arrays hold more than 2^FS_TAIL_LOG values, wide passes fold them two rounds at a
// time, four values per thread with no block barrier: a pair's weight is lo[j mod 2^10] from a
// small table of the round, and the factor hi[j >> 10], common to a CTA, multiplies the CTA's
// sums, which go to a scratch array.  All layers share each wide launch.  The last rounds of
// every layer then run in one CTA per layer (fs_tail_kernel) in shared memory, and
// fs_sums_kernel reduces the sums; fs_chain_kernel recovers each round's S(1) along the claim
// chain and writes the round polynomials.  Round polynomials hold the same field
// values as the reference's (the identities are exact), so the proofs are byte-identical.
#include <algorithm>
#include <array>
#include <cstring>

#include "prover.cuh"

namespace lgs {

namespace {

constexpr unsigned FS_THREADS = 256;
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

// The four arrays of a layer's sumcheck between kernels: A0 | U | B0 | B1, n values each (A0 is
// neither written nor read when the numerators are all one: it stays 1).
struct FsArrays {
  FsSrc src;       // before the first fold: level r+1, entries 2i, 2i+1 are element i
  const ef2* fin;  // after: the arrays (null while reading the level)
  size_t n;
  ef2 lambda;
  int ones;
  int s1;  // sum S(1) too (a layer with a zero point coordinate: the claim chain cannot divide)
};

// Rounds t (and t+1) of one layer over its whole arrays, two (or one) folds per thread.  Round t's
// pair j has weight E_{t+1}(j) = lo[j mod 2^10] hi[j >> 10]; hi is the same for a CTA's pairs, so
// it multiplies the CTA's sums.
struct FsWide {
  FsArrays in;
  ef2* fout;           // the folded arrays, (n >> rounds) values each
  ef2* part;           // [round][cta][S(0), S(1), leading coefficient]
  const ef2* lo[2];
  const ef2* hi[2];
  ef2 c[2];
  unsigned rounds, first_cta;
};

// The eq tables of one wide round: lo[i] = prod_{b<10} eq(z_{t+1+b}, bit b of i) (1024 entries)
// and hi[i] = prod_b eq(z_{t+11+b}, bit b of i) (2^(r-t-11) entries).
struct FsTable {
  const ef2* z;  // the layer's point
  ef2* lo;
  ef2* hi;
  unsigned t, r;
};

// The last rounds t0 .. r-1 of one layer in one CTA (at most 2^FS_TAIL_LOG values per array).
struct FsTail {
  FsArrays in;
  ef2* leaves;  // A0, U, B0, B1 after the last fold
  ef2* part;    // [round][S(0), S(1), leading coefficient]
  const ef2* z;
  const ef2* ch;
  unsigned r, t0;
};

// Reduction of one round: the partial sums of the kernel that ran it, into S(0), S(1), L.
struct FsRound {
  const ef2* part;  // ncta x 3
  ef2* out;         // S(0), S(1) (zero when not summed), L
  unsigned ncta;
};

// The claim chain of one layer r >= 1 (one warp, r <= 27 rounds): sigma_0 = P_r + lambda Q_r from layer r-1's
// leaves and beta_{r-1}; per round S(1) = (sigma_t - (1 - z_t) S(0)) / z_t unless it was summed,
// g(x) = K_t(x) S(x) for x = 0..3, and sigma_{t+1} = S(c_t).  (1 - z_t) S(0) + z_t S(1) = sigma_t
// is the sumcheck identity divided by C_t, so g(1) equals the reference's g(1) exactly.
struct FsChainRound {
  ef2 K[4];
  ef2 omz, invz, c, c2;  // 1 - z_t, 1 / z_t (unused when summed), c_t, c_t^2
};
struct FsChain {
  const ef2* sums;            // r x (S(0), S(1), L)
  ef2* out;                   // r x g(0..3)
  const ef2* prev;            // layer r-1's leaves: A0 A1 B0 B1 (r = 1) or A0 U B0 B1
  const FsChainRound* rounds;
  ef2 lambda, lambda_prev, beta_prev;
  unsigned r;
  int prev_direct, s1;
};

namespace {

constexpr unsigned FS_TAIL_LOG = 11;
constexpr unsigned FS_EQ_LO = 10;

struct Q4 {
  ef2 a0, u, b0, b1;
};

// One pair (lo = element 2j, hi = element 2j+1) of round t: adds w H(0), w H(1) (when S1) and w
// times the leading coefficient of H to s, and returns the element folded with c.  ONES: A0 == 1
// (numerators all one), H = B1 + B0 U.  Without S1 the round's S(1) is recovered from the claim
// chain (fs_chain_kernel), which saves three of the thirteen products.  Not inlined: a kernel
// calls it three times or more, and inlined copies of its extension-field products overflowed
// the instruction cache (ncu: "no instruction" was the top stall).
template <bool ONES, bool S1>
__device__ __noinline__ Q4 fs_pair_t(const Q4 lo, const Q4 hi, ef2 w, ef2 c, ef2 (&s)[3]) {
  Q4 o;
  const ef2 du = ef_sub(hi.u, lo.u), db0 = ef_sub(hi.b0, lo.b0), db1 = ef_sub(hi.b1, lo.b1);
  ef2 h0, h2;
  if (ONES) {
    h0 = ef_add(lo.b1, ef_mul(lo.b0, lo.u));
    h2 = ef_mul(db0, du);
    if (S1) s[1] = ef_add(s[1], ef_mul(w, ef_add(hi.b1, ef_mul(hi.b0, hi.u))));
    o.a0 = ef_one();
  } else {
    const ef2 da0 = ef_sub(hi.a0, lo.a0);
    h0 = ef_add(ef_mul(lo.a0, lo.b1), ef_mul(lo.b0, lo.u));
    h2 = ef_add(ef_mul(da0, db1), ef_mul(db0, du));
    if (S1)
      s[1] = ef_add(s[1], ef_mul(w, ef_add(ef_mul(hi.a0, hi.b1), ef_mul(hi.b0, hi.u))));
    o.a0 = ef_add(lo.a0, ef_mul(c, da0));
  }
  s[0] = ef_add(s[0], ef_mul(w, h0));
  s[2] = ef_add(s[2], ef_mul(w, h2));
  o.u = ef_add(lo.u, ef_mul(c, du));
  o.b0 = ef_add(lo.b0, ef_mul(c, db0));
  o.b1 = ef_add(lo.b1, ef_mul(c, db1));
  return o;
}
__device__ __forceinline__ Q4 fs_pair(const Q4& lo, const Q4& hi, ef2 w, ef2 c, bool ones,
                                      bool s1, ef2 (&s)[3]) {
  if (ones)
    return s1 ? fs_pair_t<true, true>(lo, hi, w, c, s) : fs_pair_t<true, false>(lo, hi, w, c, s);
  return s1 ? fs_pair_t<false, true>(lo, hi, w, c, s) : fs_pair_t<false, false>(lo, hi, w, c, s);
}

__device__ __forceinline__ Q4 arr_load(const FsArrays& a, size_t e) {
  Q4 x;
  if (a.fin) {
    x.a0 = a.ones ? ef_one() : ld_ef(a.fin + e);
    x.u = ld_ef(a.fin + a.n + e);
    x.b0 = ld_ef(a.fin + 2 * a.n + e);
    x.b1 = ld_ef(a.fin + 3 * a.n + e);
  } else {
    x.b0 = src_q(a.src, 2 * e);
    x.b1 = src_q(a.src, 2 * e + 1);
    if (a.ones) {
      x.a0 = ef_one();
      x.u = ef_add(ef_one(), ef_mul(a.lambda, x.b1));
    } else {
      x.a0 = src_p(a.src, 2 * e);
      x.u = ef_add(src_p(a.src, 2 * e + 1), ef_mul(a.lambda, x.b1));
    }
  }
  return x;
}
__device__ __forceinline__ void arr_store(ef2* out, size_t n, size_t e, const Q4& x, bool ones) {
  if (!ones) st_ef(out + e, x.a0);
  st_ef(out + n + e, x.u);
  st_ef(out + 2 * n + e, x.b0);
  st_ef(out + 3 * n + e, x.b1);
}

__device__ __forceinline__ void warp_sum3(ef2 (&s)[3]) {
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int m = 16; m; m >>= 1) s[q] = ef_add(s[q], shfl_xor_ef(s[q], m));
}

__global__ void __launch_bounds__(FS_THREADS)
    fs_tables_kernel(const FsTable* __restrict__ tabs) {
  __shared__ ef2 zs[64];
  __shared__ ef2 lo[1u << FS_EQ_LO];
  const FsTable& tb = tabs[blockIdx.x];
  const unsigned t = tb.t, r = tb.r;
  for (unsigned i = threadIdx.x; i < r; i += blockDim.x) zs[i] = ld_ef(tb.z + i);
  // lo by doubling from the high bit down: after step b, lo[i] (i < 2^(b+1)) is the product over
  // coordinates t+nlo-1-b .. t+nlo of bit order low -> high
  const unsigned nlo = r - t - 1 < FS_EQ_LO ? r - t - 1 : FS_EQ_LO;
  if (threadIdx.x == 0) lo[0] = ef_one();
  for (unsigned b = 0; b < nlo; ++b) {
    __syncthreads();
    const unsigned sz = 1u << b;
    const ef2 z = zs[t + nlo - b], nz = ef_sub(ef_one(), z);  // the new lowest coordinate
    // lo'[2m + bit] = lo[m] eq(z, bit): read all, then write (in place, top down)
    ef2 v[2][2];  // sz <= 2^(FS_EQ_LO-1) = 2 x FS_THREADS entries
#pragma unroll
    for (unsigned q = 0; q < 2; ++q) {
      const unsigned m = threadIdx.x + q * FS_THREADS;
      if (m < sz) {
        const ef2 w = lo[m];
        v[q][0] = ef_mul(w, nz);
        v[q][1] = ef_mul(w, z);
      }
    }
    __syncthreads();
#pragma unroll
    for (unsigned q = 0; q < 2; ++q) {
      const unsigned m = threadIdx.x + q * FS_THREADS;
      if (m < sz) {
        lo[2 * m] = v[q][0];
        lo[2 * m + 1] = v[q][1];
      }
    }
  }
  __syncthreads();
  for (unsigned i = threadIdx.x; i < (1u << nlo); i += blockDim.x) st_ef(tb.lo + i, lo[i]);
  const unsigned nhi = r - t - 1 - nlo;
  for (size_t i = threadIdx.x; i < ((size_t)1 << nhi); i += blockDim.x) {
    ef2 w = ef_one();
    for (unsigned b = 0; b < nhi; ++b) {
      const ef2 z = zs[t + 1 + FS_EQ_LO + b];
      w = ef_mul(w, ((i >> b) & 1) ? z : ef_sub(ef_one(), z));
    }
    st_ef(tb.hi + i, w);
  }
}

__global__ void __launch_bounds__(FS_THREADS, 2)
    fs_wide_kernel(const FsWide* __restrict__ jobs, unsigned njobs) {
  unsigned ji = 0;
  while (ji + 1 < njobs && blockIdx.x >= jobs[ji + 1].first_cta) ++ji;
  const FsWide& jb = jobs[ji];
  const bool ones = jb.in.ones != 0, s1f = jb.in.s1 != 0;
  const size_t g = (size_t)(blockIdx.x - jb.first_cta) * blockDim.x + threadIdx.x;
  const size_t nthr = jb.in.n >> jb.rounds;
  ef2 s0[3] = {ef_zero(), ef_zero(), ef_zero()};
  ef2 s1[3] = {ef_zero(), ef_zero(), ef_zero()};
  Q4 y;
  if (jb.rounds == 2) {
    const size_t e = g << 2;
    const Q4 x0 = arr_load(jb.in, e), x1 = arr_load(jb.in, e + 1);
    const Q4 x2 = arr_load(jb.in, e + 2), x3 = arr_load(jb.in, e + 3);
    const unsigned j0 = (unsigned)(2 * g) & ((1u << FS_EQ_LO) - 1);
    const Q4 f0 = fs_pair(x0, x1, ld_ef(jb.lo[0] + j0), jb.c[0], ones, s1f, s0);
    const Q4 f1 = fs_pair(x2, x3, ld_ef(jb.lo[0] + j0 + 1), jb.c[0], ones, s1f, s0);
    y = fs_pair(f0, f1, ld_ef(jb.lo[1] + (g & ((1u << FS_EQ_LO) - 1))), jb.c[1], ones, s1f,
                s1);
  } else {
    const size_t e = g << 1;
    const Q4 x0 = arr_load(jb.in, e), x1 = arr_load(jb.in, e + 1);
    y = fs_pair(x0, x1, ld_ef(jb.lo[0] + (g & ((1u << FS_EQ_LO) - 1))), jb.c[0], ones, s1f,
                s0);
  }
  arr_store(jb.fout, nthr, g, y, ones);
  // CTA sums of each round; round t's factor hi[j >> 10] is common to the CTA (256 threads cover
  // 512 or 256 consecutive pairs of an aligned block of 1024)
  __shared__ ef2 red[2][3][8];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  warp_sum3(s0);
  if (jb.rounds == 2) warp_sum3(s1);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      red[0][q][warp] = s0[q];
      red[1][q][warp] = s1[q];
    }
  __syncthreads();
  const size_t cta = blockIdx.x - jb.first_cta, ncta = nthr / FS_THREADS;
  if (threadIdx.x < 3 * jb.rounds) {
    const unsigned rd = threadIdx.x / 3, q = threadIdx.x % 3;
    ef2 v = ef_zero();
#pragma unroll
    for (int w = 0; w < 8; ++w) v = ef_add(v, red[rd][q][w]);
    const size_t g0 = cta * FS_THREADS;  // first thread of the CTA
    const size_t hj = rd == 0 ? (jb.rounds == 2 ? (g0 >> (FS_EQ_LO - 1)) : (g0 >> FS_EQ_LO))
                              : (g0 >> FS_EQ_LO);
    const ef2 h = ld_ef(jb.hi[rd] + hj);
    st_ef(jb.part + (rd * ncta + cta) * 3 + q, ef_mul(h, v));
  }
}

// Shared memory of a tail: weight tables (2^FS_TAIL_LOG entries), the folded elements after the
// first round (2^(FS_TAIL_LOG-1)), per-warp round sums (FS_TAIL_LOG x 16 warps x 3).
constexpr size_t FS_TAIL_SMEM = ((size_t)1 << FS_TAIL_LOG) * sizeof(ef2) +
                                ((size_t)1 << (FS_TAIL_LOG - 1)) * sizeof(Q4) +
                                (size_t)FS_TAIL_LOG * 16 * 3 * sizeof(ef2);
constexpr unsigned FS_TAIL_THREADS = 512;  // latency-bound: as many warps as the registers allow

__global__ void __launch_bounds__(FS_TAIL_THREADS) fs_tail_kernel(const FsTail* __restrict__ jobs) {
  extern __shared__ ef2 fs_sm[];
  ef2* wt = fs_sm;  // W_tau at offset 2^(nb - tau - 1) - 1
  Q4* xs = reinterpret_cast<Q4*>(fs_sm + (1u << FS_TAIL_LOG));
  ef2* acc = fs_sm + (1u << FS_TAIL_LOG) + 4 * (1u << (FS_TAIL_LOG - 1));  // [tau][warp][3]
  const FsTail& jb = jobs[blockIdx.x];
  const unsigned t0 = jb.t0, nb = jb.r - t0;
  const bool ones = jb.in.ones != 0, s1f = jb.in.s1 != 0;
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;

  // W_{nb-1} = [1]; W_tau[2m + b] = W_{tau+1}[m] eq(z_{t0+tau+1}, b): the weight of pair jl in
  // round t0+tau is E_{t0+tau+1}(jl).
  if (threadIdx.x == 0) wt[0] = ef_one();
  for (int tau = (int)nb - 2; tau >= 0; --tau) {
    __syncthreads();
    const unsigned sz = 1u << (nb - tau - 1), prev = (sz >> 1) - 1, off = sz - 1;
    const ef2 z1 = ld_ef(jb.z + t0 + tau + 1), z0 = ef_sub(ef_one(), z1);
    for (unsigned i = threadIdx.x; i < sz; i += blockDim.x)
      wt[off + i] = ef_mul(wt[prev + (i >> 1)], (i & 1) ? z1 : z0);
  }
  __syncthreads();

  auto warp_acc = [&](ef2 (&s)[3], unsigned tau) {  // per-warp sums, no block barrier
    warp_sum3(s);
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < 3; ++q) acc[(tau * nw + warp) * 3 + q] = s[q];
  };
  {  // round t0 from global memory
    const unsigned np = 1u << (nb - 1);
    const ef2 c = ld_ef(jb.ch + t0);
    ef2 s[3] = {ef_zero(), ef_zero(), ef_zero()};
    for (unsigned jl = threadIdx.x; jl < np; jl += blockDim.x) {
      const Q4 lo = arr_load(jb.in, 2 * jl), hi = arr_load(jb.in, 2 * jl + 1);
      xs[jl] = fs_pair(lo, hi, wt[np - 1 + jl], c, ones, s1f, s);
    }
    warp_acc(s, 0);
  }
  // rounds with more pairs than one warp: exchange through shared memory with barriers
  unsigned tau = 1;
  for (; tau < nb && (1u << (nb - tau - 1)) > 32; ++tau) {
    const unsigned np = 1u << (nb - tau - 1);
    const ef2 c = ld_ef(jb.ch + t0 + tau);
    ef2 s[3] = {ef_zero(), ef_zero(), ef_zero()};
    Q4 o[2];
    __syncthreads();
#pragma unroll
    for (unsigned q = 0; q < 2; ++q) {
      const unsigned jl = threadIdx.x + q * blockDim.x;
      if (jl < np)
        o[q] = fs_pair(xs[2 * jl], xs[2 * jl + 1], wt[np - 1 + jl], c, ones, s1f, s);
    }
    __syncthreads();
#pragma unroll
    for (unsigned q = 0; q < 2; ++q) {
      const unsigned jl = threadIdx.x + q * blockDim.x;
      if (jl < np) xs[jl] = o[q];
    }
    warp_acc(s, tau);
  }
  __syncthreads();
  // the rest in warp 0 (the other warps' sums of these rounds are zero)
  for (; tau < nb; ++tau) {
    const unsigned np = 1u << (nb - tau - 1);
    ef2 s[3] = {ef_zero(), ef_zero(), ef_zero()};
    if (warp == 0) {
      const ef2 c = ld_ef(jb.ch + t0 + tau);
      Q4 o;
      if (lane < np)
        o = fs_pair(xs[2 * lane], xs[2 * lane + 1], wt[np - 1 + lane], c, ones, s1f, s);
      __syncwarp();
      if (lane < np) xs[lane] = o;
      __syncwarp();
    }
    warp_acc(s, tau);
  }
  __syncthreads();
  for (unsigned i = threadIdx.x; i < nb * 3; i += blockDim.x) {
    const unsigned tt = i / 3, q = i % 3;
    ef2 v = ef_zero();
    for (unsigned w = 0; w < nw; ++w) v = ef_add(v, acc[(tt * nw + w) * 3 + q]);
    st_ef(jb.part + i, v);
  }
  if (threadIdx.x == 0) {
    const Q4 x = xs[0];
    st_ef(jb.leaves + 0, x.a0);
    st_ef(jb.leaves + 1, x.u);
    st_ef(jb.leaves + 2, x.b0);
    st_ef(jb.leaves + 3, x.b1);
  }
}

// Sums the partial sums of each round: one CTA per round.
__global__ void __launch_bounds__(FS_THREADS) fs_sums_kernel(const FsRound* __restrict__ rounds) {
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
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 3; ++q) st_ef(rd.out + q, s[q]);
}

// g(x) = K(x) S(x) with S quadratic: S(2) = -S(0) + 2 S(1) + 2 L, S(3) = -2 S(0) + 3 S(1) + 6 L
// (L the leading coefficient).  One warp per layer (see FsChain): lane t holds round t's sums and
// constants (loaded at once), the chain passes sigma from lane to lane, and every lane then writes
// its own round polynomial.
__global__ void __launch_bounds__(32) fs_chain_kernel(const FsChain* __restrict__ chains) {
  const FsChain& ch = chains[blockIdx.x];
  const unsigned lane = threadIdx.x, r = ch.r;
  const bool act = lane < r;
  FsChainRound rd{};
  ef2 s0 = ef_zero(), s1 = ef_zero(), l = ef_zero();
  if (act) {
    rd = ch.rounds[lane];
    s0 = ld_ef(ch.sums + 3 * lane);
    s1 = ld_ef(ch.sums + 3 * lane + 1);
    l = ld_ef(ch.sums + 3 * lane + 2);
  }
  ef2 sigma = ef_zero();
  if (lane == 0) {
    const ef2 a0 = ld_ef(ch.prev), b0 = ld_ef(ch.prev + 2), b1 = ld_ef(ch.prev + 3);
    const ef2 a1 = ch.prev_direct ? ld_ef(ch.prev + 1)
                                  : ef_sub(ld_ef(ch.prev + 1), ef_mul(ch.lambda_prev, b1));
    const ef2 P = ef_add(a0, ef_mul(ch.beta_prev, ef_sub(a1, a0)));
    const ef2 Q = ef_add(b0, ef_mul(ch.beta_prev, ef_sub(b1, b0)));
    sigma = ef_add(P, ef_mul(ch.lambda, Q));
  }
  // sigma_{t+1} = S(c) = S(0) + (S(1) - S(0) - L) c + L c^2 is affine in sigma_t: with
  // S(1) = (sigma_t - (1 - z) S(0)) / z it is beta_t + gamma_t sigma_t, gamma_t = c / z; with S(1)
  // summed, gamma_t = 0.  Only the one product gamma_t sigma_t per round is sequential.
  const ef2 base = ef_add(ef_sub(s0, ef_mul(ef_add(s0, l), rd.c)), ef_mul(l, rd.c2));
  ef2 gamma = ef_zero(), beta;
  if (ch.s1) {
    beta = ef_add(base, ef_mul(s1, rd.c));
  } else {
    gamma = ef_mul(rd.invz, rd.c);
    beta = ef_sub(base, ef_mul(gamma, ef_mul(rd.omz, s0)));
  }
  ef2 mine = ef_zero();  // sigma_lane
  for (unsigned t = 0; t < r; ++t) {
    ef2 next = ef_zero();
    if (lane == t) {
      mine = sigma;
      next = ef_add(beta, ef_mul(gamma, sigma));
    }
    sigma = ef_make(__shfl_sync(0xffffffffu, next.c0, t), __shfl_sync(0xffffffffu, next.c1, t));
  }
  if (act && !ch.s1) s1 = ef_mul(ef_sub(mine, ef_mul(rd.omz, s0)), rd.invz);
  if (!act) return;
  const ef2 two_s1 = ef_add(s1, s1), two_l = ef_add(l, l);
  const ef2 s2 = ef_sub(ef_add(two_s1, two_l), s0);
  const ef2 s3 = ef_sub(ef_add(ef_add(two_s1, s1), ef_add(ef_add(two_l, two_l), two_l)),
                        ef_add(s0, s0));
  st_ef(ch.out + 4 * lane + 0, ef_mul(rd.K[0], s0));
  st_ef(ch.out + 4 * lane + 1, ef_mul(rd.K[1], s1));
  st_ef(ch.out + 4 * lane + 2, ef_mul(rd.K[2], s2));
  st_ef(ch.out + 4 * lane + 3, ef_mul(rd.K[3], s3));
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

// The device plan of one fraction-sum proof: its challenges, device buffers, the parameter blob
// its kernels read, and where its values land in the staging area.
struct FsPlan {
  unsigned k = 0;
  uint64_t f0 = 0;              // fields cursor at the start
  std::vector<ef2> lambda, beta;
  std::vector<std::vector<ef2>> z, ch;
  size_t stage_off = 0;         // EF offset of this proof's values in the staging area
  size_t round_off = 0;         // EF offset of the round polynomials (within the staging)
  size_t stage_elems = 0;
  FsSrc in{};
  ef2* stage = nullptr;
  ef2* P = nullptr;
  ef2* Q = nullptr;
  uint8_t* d_up = nullptr;
  std::vector<uint8_t> blob;    // z / challenges, tables, wide jobs (launch by launch), tails,
                                // rounds
  size_t up_tables = 0, up_wide = 0, up_tails = 0, up_rounds = 0, up_chains = 0, up_crounds = 0;
  size_t nrounds = 0;
  unsigned ntables = 0, ntails = 0, nchains = 0;
  std::vector<unsigned> pass_jobs, pass_ctas;
};

static size_t fs_fields_needed(unsigned k) { return (size_t)k * (k + 3) / 2; }

// Plans one fraction-sum proof of 2^k inputs: challenges, device buffers (from the arena) and the
// parameter blob.  Its values land in `stage` (device) at stage_off: num, den, level-1 entries
// (6 EF), then per layer r >= 1 the leaves (A0, U, B0, B1), then the round polynomials layer by
// layer.
static void fs_plan(lgs_ctx* c, const FsSrc& in, unsigned k, const u64* fields, size_t nfields,
                    uint64_t f0, ef2* stage, size_t stage_off, FsPlan* plan) {
  Arena& ar = c->arena;
  if (k > FS_MAX_K) throw ShapeError("frac_sum: at most 2^28 fractions");
  const size_t need = fs_fields_needed(k);
  if (f0 > nfields || nfields - f0 < need) throw OracleError("oracle exhausted (fields)");
  plan->k = k;
  plan->f0 = f0;
  plan->in = in;
  plan->stage = stage;
  plan->stage_off = stage_off;
  auto F = [&](size_t i) {
    return ef_make(gl_canon(fields[2 * (f0 + i)]), gl_canon(fields[2 * (f0 + i) + 1]));
  };
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
  plan->nrounds = nrounds;
  plan->round_off = stage_off + 6 + 4 * (k ? k - 1 : 0);
  plan->stage_elems = k ? 6 + 4 * (k - 1) + 4 * nrounds : 2;
  if (k == 0) return;

  const size_t nlev = ((size_t)1 << k) - 1;  // levels 0 .. k-1
  ef2* P = plan->P = ar.get<ef2>(nlev);
  ef2* Q = plan->Q = ar.get<ef2>(nlev);
  auto level = [&](unsigned s) -> FsSrc {
    if (s == k) return in;
    return FsSrc{P + ((size_t)1 << s) - 1, Q + ((size_t)1 << s) - 1, ef_zero(), 0};
  };

  std::vector<std::vector<FsWide>> wide;  // per wide launch
  std::vector<FsTable> tables;
  std::vector<FsTail> tails;
  std::vector<FsRound> rounds;
  std::vector<FsChain> chains;
  std::vector<FsChainRound> crounds;
  std::vector<ef2> zc;  // z_r then ch_r for every layer r >= 1
  std::vector<size_t> zoff(k, 0);
  for (unsigned r = 1; r < k; ++r) {
    zoff[r] = zc.size();
    zc.insert(zc.end(), plan->z[r].begin(), plan->z[r].end());
    zc.insert(zc.end(), plan->ch[r].begin(), plan->ch[r].end());
  }
  // device pointers into the blob are fixed once its layout is: count the records first
  size_t n_wide = 0, n_tab = 0;
  for (unsigned r = 1; r < k; ++r)
    for (size_t n = (size_t)1 << r; n > ((size_t)1 << FS_TAIL_LOG);) {
      const unsigned rr = n >= ((size_t)4 << FS_TAIL_LOG) ? 2 : 1;
      ++n_wide;
      n_tab += rr;
      n >>= rr;
    }
  size_t up_bytes = ceil256(zc.size() * sizeof(ef2));
  plan->up_tables = up_bytes;
  up_bytes += ceil256(n_tab * sizeof(FsTable));
  plan->up_wide = up_bytes;
  up_bytes += ceil256(n_wide * sizeof(FsWide));
  plan->up_tails = up_bytes;
  up_bytes += ceil256((k - 1) * sizeof(FsTail));
  plan->up_rounds = up_bytes;
  up_bytes += ceil256(nrounds * sizeof(FsRound));
  plan->up_chains = up_bytes;
  up_bytes += ceil256((k - 1) * sizeof(FsChain));
  plan->up_crounds = up_bytes;
  up_bytes += ceil256(nrounds * sizeof(FsChainRound));
  uint8_t* d_up = plan->d_up = ar.get<uint8_t>(up_bytes);
  std::vector<uint8_t>& h_up = plan->blob;
  h_up.assign(up_bytes, 0);
  std::memcpy(h_up.data(), zc.data(), zc.size() * sizeof(ef2));
  const ef2* d_zc = (const ef2*)d_up;

  // 1 / z_t for every round (one inversion, Montgomery's batch trick); a layer with a zero
  // coordinate sums S(1) instead (its chain cannot divide)
  std::vector<int> layer_s1(k, 0);
  std::vector<ef2> invz;
  {
    std::vector<ef2> pre;
    ef2 acc = ef_one();
    for (unsigned r = 1; r < k; ++r)
      for (const ef2& zt : plan->z[r]) {
        if (ef_eq(zt, ef_zero())) layer_s1[r] = 1;
        pre.push_back(acc);
        if (!ef_eq(zt, ef_zero())) acc = ef_mul(acc, zt);
      }
    invz.assign(pre.size(), ef_zero());
    ef2 inv = ef_inv(acc);  // acc is a product of nonzero values
    size_t i = pre.size();
    for (unsigned r = k - 1; r >= 1; --r)
      for (unsigned t = r; t-- > 0;) {
        const ef2 zt = plan->z[r][t];
        --i;
        if (ef_eq(zt, ef_zero())) continue;
        invz[i] = ef_mul(inv, pre[i]);
        inv = ef_mul(inv, zt);
      }
  }
  ef2* sums = ar.get<ef2>(3 * nrounds);
  const FsChainRound* d_crounds = (const FsChainRound*)(d_up + plan->up_crounds);
  size_t round_pos = plan->round_off, round_idx = 0;
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
    auto add_round = [&](unsigned t, const ef2* part, unsigned nparts) {
      FsRound rd{};
      rd.part = part;
      rd.out = sums + 3 * (round_idx + t);
      rd.ncta = nparts;
      rounds.push_back(rd);
    };
    FsChain chn{};
    chn.sums = sums + 3 * round_idx;
    chn.out = stage + round_pos;
    chn.prev = r == 1 ? stage + stage_off + 2 : stage + stage_off + 6 + 4 * (r - 2);
    chn.rounds = d_crounds + round_idx;
    chn.lambda = plan->lambda[r];
    chn.lambda_prev = plan->lambda[r - 1];
    chn.beta_prev = plan->beta[r - 1];
    chn.r = r;
    chn.prev_direct = r == 1 ? 1 : 0;
    chn.s1 = layer_s1[r];
    chains.push_back(chn);
    for (unsigned t = 0; t < r; ++t) {
      FsChainRound cr{};
      for (int x = 0; x < 4; ++x) cr.K[x] = K[t][x];
      cr.omz = ef_sub(ef_one(), plan->z[r][t]);
      cr.invz = invz[round_idx + t];
      cr.c = plan->ch[r][t];
      cr.c2 = ef_mul(cr.c, cr.c);
      crounds.push_back(cr);
    }
    FsArrays cur{level(r + 1), nullptr, (size_t)1 << r, plan->lambda[r],
                 (r + 1 == k && in.p == nullptr) ? 1 : 0, layer_s1[r]};
    unsigned t = 0, pass = 0;
    while (cur.n > ((size_t)1 << FS_TAIL_LOG)) {
      FsWide w{};
      w.in = cur;
      w.rounds = cur.n >= ((size_t)4 << FS_TAIL_LOG) ? 2 : 1;
      const size_t nout = cur.n >> w.rounds, nctas = nout / FS_THREADS;
      w.fout = ar.get<ef2>(4 * nout);
      w.part = ar.get<ef2>(w.rounds * nctas * 3);
      for (unsigned q = 0; q < w.rounds; ++q) {
        FsTable tb{};
        tb.z = z;
        tb.t = t + q;
        tb.r = r;
        tb.lo = ar.get<ef2>((size_t)1 << FS_EQ_LO);
        tb.hi = ar.get<ef2>((size_t)1 << (r - (t + q) - 1 - FS_EQ_LO));
        tables.push_back(tb);
        w.lo[q] = tb.lo;
        w.hi[q] = tb.hi;
        w.c[q] = plan->ch[r][t + q];
        add_round(t + q, w.part + q * nctas * 3, (unsigned)nctas);
      }
      if (wide.size() <= pass) wide.resize(pass + 1);
      wide[pass].push_back(w);
      cur.fin = w.fout;
      cur.n = nout;
      t += w.rounds;
      ++pass;
    }
    FsTail tl{};
    tl.in = cur;
    tl.leaves = stage + stage_off + 6 + 4 * (r - 1);
    tl.part = ar.get<ef2>((size_t)(r - t) * 3);
    tl.z = z;
    tl.ch = chp;
    tl.r = r;
    tl.t0 = t;
    tails.push_back(tl);
    for (unsigned q = t; q < r; ++q) add_round(q, tl.part + (size_t)(q - t) * 3, 1);
    round_pos += 4 * (size_t)r;
    round_idx += r;
  }
  std::memcpy(h_up.data() + plan->up_tables, tables.data(), tables.size() * sizeof(FsTable));
  plan->ntables = (unsigned)tables.size();
  size_t o = plan->up_wide;
  for (auto& pj : wide) {
    unsigned first = 0;
    for (auto& w : pj) {
      w.first_cta = first;
      first += (unsigned)((w.in.n >> w.rounds) / FS_THREADS);
    }
    std::memcpy(h_up.data() + o, pj.data(), pj.size() * sizeof(FsWide));
    o += pj.size() * sizeof(FsWide);
    plan->pass_jobs.push_back((unsigned)pj.size());
    plan->pass_ctas.push_back(first);
  }
  std::memcpy(h_up.data() + plan->up_tails, tails.data(), tails.size() * sizeof(FsTail));
  plan->ntails = (unsigned)tails.size();
  std::memcpy(h_up.data() + plan->up_rounds, rounds.data(), rounds.size() * sizeof(FsRound));
  std::memcpy(h_up.data() + plan->up_chains, chains.data(), chains.size() * sizeof(FsChain));
  std::memcpy(h_up.data() + plan->up_crounds, crounds.data(),
              crounds.size() * sizeof(FsChainRound));
  plan->nchains = (unsigned)chains.size();
}

// Enqueues a planned proof on st; `pinned` is page-locked host memory holding nothing else for
// plan->blob.size() bytes until the stream has passed the copy.
static void fs_launch(const FsPlan& pl, uint8_t* pinned, cudaStream_t st) {
  const unsigned k = pl.k;
  if (k == 0) {
    fs_single_kernel<<<1, 32, 0, st>>>(pl.in, pl.stage + pl.stage_off);
    LGS_LAUNCH_CHECK();
    return;
  }
  std::memcpy(pinned, pl.blob.data(), pl.blob.size());
  LGS_CUDA(cudaMemcpyAsync(pl.d_up, pinned, pl.blob.size(), cudaMemcpyHostToDevice, st));
  ef2* P = pl.P;
  ef2* Q = pl.Q;
  if (pl.ntables) {
    fs_tables_kernel<<<pl.ntables, FS_THREADS, 0, st>>>((const FsTable*)(pl.d_up + pl.up_tables));
    LGS_LAUNCH_CHECK();
  }
  {
    unsigned S = k;
    FsSrc src = pl.in;
    while (S > 0) {
      const unsigned T = std::min(S, FS_BUILD_T);
      const size_t smem = 2 * ((size_t)1 << T) * sizeof(ef2);
      fs_build_kernel<<<(unsigned)((size_t)1 << (S - T)), FS_THREADS, smem, st>>>(src, S, T, P, Q);
      LGS_LAUNCH_CHECK();
      S -= T;
      src = FsSrc{P + ((size_t)1 << S) - 1, Q + ((size_t)1 << S) - 1, ef_zero(), 0};
    }
  }
  const FsWide* dw = (const FsWide*)(pl.d_up + pl.up_wide);
  for (size_t pi = 0; pi < pl.pass_jobs.size(); ++pi) {
    fs_wide_kernel<<<pl.pass_ctas[pi], FS_THREADS, 0, st>>>(dw, pl.pass_jobs[pi]);
    LGS_LAUNCH_CHECK();
    dw += pl.pass_jobs[pi];
  }
  if (pl.ntails) {
    fs_tail_kernel<<<pl.ntails, FS_TAIL_THREADS, FS_TAIL_SMEM, st>>>(
        (const FsTail*)(pl.d_up + pl.up_tails));
    LGS_LAUNCH_CHECK();
  }
  if (pl.nrounds) {
    fs_sums_kernel<<<(unsigned)pl.nrounds, FS_THREADS, 0, st>>>(
        (const FsRound*)(pl.d_up + pl.up_rounds));
    LGS_LAUNCH_CHECK();
  }
  const FsSrc l1 = k == 1 ? pl.in : FsSrc{P + 1, Q + 1, ef_zero(), 0};
  fs_root_kernel<<<1, 32, 0, st>>>(l1, P, Q, pl.stage + pl.stage_off);
  LGS_LAUNCH_CHECK();
  if (pl.nchains) {  // after the root kernel: layer 1's chain starts from level 1's entries
    fs_chain_kernel<<<pl.nchains, 32, 0, st>>>((const FsChain*)(pl.d_up + pl.up_chains));
    LGS_LAUNCH_CHECK();
  }
}

static void fs_kernel_attrs() {
  LGS_CUDA(cudaFuncSetAttribute(fs_tail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)FS_TAIL_SMEM));
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
  fs_plan(c, in, k, fields, nfields, *cursor, stage, 0, &pl);
  fs_kernel_attrs();
  c->up.reserve(pl.blob.size());
  fs_launch(pl, c->up.as<uint8_t>(), st);
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
  fs_plan(c, FsSrc{nullptr, da, alpha, 1}, kq, fields, nfields, f0 + 1, stage, 0, &pq);
  fs_plan(c, FsSrc{de, dt, alpha, 1}, kt, fields, nfields, f0 + 1 + fs_fields_needed(kq), stage,
          eq_n, &ptab);
  fs_kernel_attrs();
  const size_t qb = ceil256(pq.blob.size());
  c->up.reserve(qb + ptab.blob.size());
  fs_launch(pq, c->up.as<uint8_t>(), st);
  fs_launch(ptab, c->up.as<uint8_t>() + qb, sd);
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
