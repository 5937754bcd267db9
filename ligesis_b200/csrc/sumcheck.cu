// Product sumcheck prover (utils/src/sumcheck.rs:37-84) on the device.
//
// Round t sends g_t(q) = sum_{i < half} prod_j (lo_j + q (hi_j - lo_j)), q = 0..d, with
// lo = P[i], hi = P[i + half] (the HIGH variable is bound first), then folds every factor with
// the round challenge r_t: P[i] = P[i] + r_t (P[i + half] - P[i]).  All challenges come from the
// pre-drawn oracle (utils/src/oracle.rs:10-64), so no round depends on the host: the fold of
// round t-1 is fused into the evaluation pass of round t (each thread owns the quadruple
// i, i + half, i + 2 half, i + 3 half, so the in-place fold has no races), per-CTA partial sums
// go to a scratch array, and a last kernel reduces them into the round polynomials.  Once the
// vectors are short (1024 entries, 512 for three stored factors), one CTA loads them into shared
// memory and finishes the remaining rounds there.
//
// Binary variant (the B_I check of pcs/src/ligesis.rs:423-428, factors [b, b - 1, eq]): the
// middle factor is always the first minus one (folding is affine), so only b and eq are stored
// and folded; the products, round messages and final evaluations are those of the 3-factor run.
#include "kernels.cuh"

namespace lgs {

namespace {
constexpr unsigned SC_THREADS = 256;
constexpr unsigned SC_TAIL_THREADS = 128;

__device__ __forceinline__ ef2 shfl_xor_ef(ef2 v, int m) {
  ef2 r;
  r.c0 = __shfl_xor_sync(0xffffffffu, v.c0, m);
  r.c1 = __shfl_xor_sync(0xffffffffu, v.c1, m);
  return r;
}

// Sum D+1 EF values over the CTA; result valid in thread 0.  `red` holds (D+1) * 32 entries.
template <int D>
__device__ void block_reduce(ef2 (&s)[D + 1], ef2* red) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q <= D; ++q)
#pragma unroll
    for (int m = 16; m; m >>= 1) s[q] = ef_add(s[q], shfl_xor_ef(s[q], m));
  if (lane == 0)
#pragma unroll
    for (int q = 0; q <= D; ++q) red[q * 32 + warp] = s[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q <= D; ++q) {
      ef2 v = lane < nw ? red[q * 32 + lane] : ef_zero();
#pragma unroll
      for (int m = 16; m; m >>= 1) v = ef_add(v, shfl_xor_ef(v, m));
      s[q] = v;
    }
  }
  __syncthreads();
}

// Stored factor count: the binary variant keeps [b, eq] for the logical [b, b - 1, eq].
template <int D, bool BIN>
struct Fac {
  static constexpr int S = BIN ? D - 1 : D;
  // vectors at most this long finish in one CTA (in at most 48 KB of static shared memory)
  static constexpr unsigned TAIL = S >= 3 ? 512 : 1024;
};

// Add prod_j (lo_j + q (hi_j - lo_j)) for q = 0..D to s, from the stored factors.  skip1: leave
// out q = 1 (the round's g(1) is then recovered from the running claim, g(1) = claim - g(0)).
template <int D, bool BIN>
__device__ __forceinline__ void accumulate_pair(const ef2* lo, const ef2* hi, ef2 (&s)[D + 1],
                                                bool skip1) {
  constexpr int S = Fac<D, BIN>::S;
  ef2 v[S], df[S];
#pragma unroll
  for (int j = 0; j < S; ++j) v[j] = lo[j], df[j] = ef_sub(hi[j], lo[j]);
#pragma unroll
  for (int q = 0; q <= D; ++q) {
    if (q != 1 || !skip1) {
      ef2 p;
      if (BIN) {
        p = ef_mul(v[0], ef_sub(v[0], ef_one()));  // b (b - 1)
#pragma unroll
        for (int j = 1; j < S; ++j) p = ef_mul(p, v[j]);
      } else {
        p = v[0];
#pragma unroll
        for (int j = 1; j < S; ++j) p = ef_mul(p, v[j]);
      }
      s[q] = ef_add(s[q], p);
    }
    if (q < D)
#pragma unroll
      for (int j = 0; j < S; ++j) v[j] = (q == 0) ? hi[j] : ef_add(v[j], df[j]);
  }
}

// One pair's contributions, out of line: inlined, the pair arithmetic appears three times in a
// two-round pass (and in the one-round and tail kernels), and those copies overflowed the
// instruction cache (warps stalled on instruction fetch).  Small structs by value keep the
// operands in registers across the call.
template <int S>
struct FacVals {
  ef2 v[S];
};
template <int D>
struct PairSums {
  ef2 s[D + 1];
};
template <int D, bool BIN>
__device__ __noinline__ PairSums<D> pair_sums(FacVals<Fac<D, BIN>::S> lo,
                                              FacVals<Fac<D, BIN>::S> hi, bool skip1) {
  PairSums<D> r;
#pragma unroll
  for (int q = 0; q <= D; ++q) r.s[q] = ef_zero();
  accumulate_pair<D, BIN>(lo.v, hi.v, r.s, skip1);
  return r;
}
template <int D, bool BIN>
__device__ __forceinline__ void add_pair(const ef2* lo, const ef2* hi, ef2 (&s)[D + 1],
                                         bool skip1) {
  constexpr int S = Fac<D, BIN>::S;
  FacVals<S> a, b;
#pragma unroll
  for (int j = 0; j < S; ++j) a.v[j] = lo[j], b.v[j] = hi[j];
  const PairSums<D> r = pair_sums<D, BIN>(a, b, skip1);
#pragma unroll
  for (int q = 0; q <= D; ++q) s[q] = ef_add(s[q], r.s[q]);
}

// g(r) for the degree-D round polynomial given by its values g(0..D) (Lagrange on 0..D).
template <int D>
__device__ ef2 interp_at(const ef2* g, ef2 r) {
  const u64 inv2 = 0x7FFFFFFF80000001ULL, inv6 = 0xD555555480000001ULL;
  const ef2 r1 = ef_sub(r, ef_from(1)), r2 = ef_sub(r, ef_from(2));
  if (D == 1) return ef_add(g[0], ef_mul(r, ef_sub(g[1], g[0])));
  if (D == 2) {
    const ef2 l0 = ef_scale(ef_mul(r1, r2), inv2);
    const ef2 l1 = ef_sub(ef_zero(), ef_mul(r, r2));
    const ef2 l2 = ef_scale(ef_mul(r, r1), inv2);
    return ef_add(ef_add(ef_mul(g[0], l0), ef_mul(g[1], l1)), ef_mul(g[2], l2));
  }
  const ef2 r3 = ef_sub(r, ef_from(3));
  const ef2 r12 = ef_mul(r1, r2), rr1 = ef_mul(r, r1);
  const ef2 l0 = ef_sub(ef_zero(), ef_scale(ef_mul(r12, r3), inv6));
  const ef2 l1 = ef_scale(ef_mul(ef_mul(r, r2), r3), inv2);
  const ef2 l2 = ef_sub(ef_zero(), ef_scale(ef_mul(rr1, r3), inv2));
  const ef2 l3 = ef_scale(ef_mul(rr1, r2), inv6);
  return ef_add(ef_add(ef_mul(g[0], l0), ef_mul(g[1], l1)),
                ef_add(ef_mul(g[2], l2), ef_mul(g[3], l3)));
}

template <int S>
struct Polys {
  ef2* p[S];
};

// One round over `half` pairs.  If `fold`, the vectors still hold 4*half entries from the
// previous round and are folded with r first (results written back to [0, 2*half)).
template <int D, bool BIN>
__global__ void __launch_bounds__(SC_THREADS)
    sc_round_kernel(Polys<Fac<D, BIN>::S> P, size_t half, int fold, const ef2* __restrict__ rptr,
                    ef2* __restrict__ partial) {
  const bool skip1 = fold != 0;  // every round but the first: g(1) comes from the claim
  constexpr int S = Fac<D, BIN>::S;
  __shared__ ef2 red[(D + 1) * 32];
  ef2 s[D + 1];
#pragma unroll
  for (int q = 0; q <= D; ++q) s[q] = ef_zero();
  const ef2 r = fold ? *rptr : ef_zero();
  const size_t len = 2 * half;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < half;
       i += (size_t)gridDim.x * blockDim.x) {
    ef2 lo[S], hi[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
      ef2* p = P.p[j];
      if (fold) {
        lo[j] = ef_lerp(p[i], p[i + len], r);
        hi[j] = ef_lerp(p[i + half], p[i + half + len], r);
        p[i] = lo[j];
        p[i + half] = hi[j];
      } else {
        lo[j] = p[i];
        hi[j] = p[i + half];
      }
    }
    add_pair<D, BIN>(lo, hi, s, skip1);
  }
  block_reduce<D>(s, red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q <= D; ++q) partial[(size_t)blockIdx.x * (D + 1) + q] = s[q];
}

// Rounds t and t+1 in one pass.  On entry the vectors hold 2*len entries still to be folded with
// r_{t-1} (fold != 0), or len entries (fold == 0, t == 0).  Thread i < len/4 owns the elements
// i + m len/4 (m = 0..3) of the folded vectors: round t's pairs are (i, i + len/2) and
// (i + len/4, i + 3 len/4); folded with r_t they become elements i and i + len/4, which are round
// t+1's pair and are stored there, to be folded with r_{t+1} by the next pass.  Each position the
// thread writes is read only by the same thread, so the update in place has no races.  Against
// two single-round passes this reads a third less, writes two thirds less and halves the
// launches.  Round t's partials use the grid of round t+1; the slots a one-round pass would have
// used beyond it (nb_t of them) are zeroed.
template <int D, bool BIN>
__global__ void __launch_bounds__(SC_THREADS, 2)
    sc_round2_kernel(Polys<Fac<D, BIN>::S> P, size_t len, int fold, const ef2* __restrict__ rprev,
                     const ef2* __restrict__ rt, ef2* __restrict__ part_t,
                     ef2* __restrict__ part_t1, unsigned nb_t) {
  constexpr int S = Fac<D, BIN>::S;
  __shared__ ef2 red[(D + 1) * 32];
  const bool skip1 = fold != 0;  // round t's g(1) comes from the claim unless t == 0
  ef2 s0[D + 1], s1[D + 1];
#pragma unroll
  for (int q = 0; q <= D; ++q) s0[q] = ef_zero(), s1[q] = ef_zero();
  const ef2 ra = fold ? *rprev : ef_zero(), rb = *rt;
  const size_t qlen = len >> 2;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < qlen;
       i += (size_t)gridDim.x * blockDim.x) {
    // The two pairs of round t one after the other (fewer values live at once): pair m is
    // (i + m qlen, i + (m + 2) qlen), folded with r_t into element i + m qlen.
    ef2 y[2][S];
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      ef2 lo[S], hi[S];
#pragma unroll
      for (int j = 0; j < S; ++j) {
        const ef2* p = P.p[j];
        const size_t x = i + m * qlen, xh = x + 2 * qlen;
        lo[j] = fold ? ef_lerp(p[x], p[x + len], ra) : p[x];
        hi[j] = fold ? ef_lerp(p[xh], p[xh + len], ra) : p[xh];
      }
      add_pair<D, BIN>(lo, hi, s0, skip1);
#pragma unroll
      for (int j = 0; j < S; ++j) {
        y[m][j] = ef_lerp(lo[j], hi[j], rb);
        P.p[j][i + m * qlen] = y[m][j];
      }
    }
    add_pair<D, BIN>(y[0], y[1], s1, true);
  }
  block_reduce<D>(s0, red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q <= D; ++q) part_t[(size_t)blockIdx.x * (D + 1) + q] = s0[q];
  block_reduce<D>(s1, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q <= D; ++q) part_t1[(size_t)blockIdx.x * (D + 1) + q] = s1[q];
    const unsigned extra = blockIdx.x + gridDim.x;
    if (extra < nb_t)
#pragma unroll
      for (int q = 0; q <= D; ++q) part_t[(size_t)extra * (D + 1) + q] = ef_zero();
  }
}

// Round 0 of the binary check [b, b - 1, eq] with b in {0, 1}: over a pair, b(q) (b(q) - 1) is 0
// at q = 0, 1, and 2 resp. 6 at q = 2, 3 exactly when lo != hi (b(q) = q or 1 - q), so the round
// is g(0) = g(1) = 0, g(2) = 2 sum eq(2), g(3) = 6 sum eq(3) over the pairs with lo != hi.
__global__ void __launch_bounds__(SC_THREADS)
    sc_bin_round0_kernel(const ef2* __restrict__ b, const ef2* __restrict__ eq, size_t half,
                         ef2* __restrict__ partial) {
  __shared__ ef2 red[4 * 32];
  ef2 s[4] = {ef_zero(), ef_zero(), ef_zero(), ef_zero()};
  const u64* bc = (const u64*)b;  // c0 of b[i] at bc[2 i]
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < half;
       i += (size_t)gridDim.x * blockDim.x) {
    if (bc[2 * i] != bc[2 * (i + half)]) {
      const ef2 lo = eq[i], hi = eq[i + half];
      const ef2 d = ef_sub(hi, lo), e2 = ef_add(hi, d);
      s[2] = ef_add(s[2], e2);
      s[3] = ef_add(s[3], ef_add(e2, d));
    }
  }
  block_reduce<3>(s, red);
  if (threadIdx.x == 0) {
    partial[(size_t)blockIdx.x * 4 + 0] = ef_zero();
    partial[(size_t)blockIdx.x * 4 + 1] = ef_zero();
    partial[(size_t)blockIdx.x * 4 + 2] = ef_scale(s[2], 2);
    partial[(size_t)blockIdx.x * 4 + 3] = ef_scale(s[3], 6);
  }
}

// Lagrange weights of the nodes 0..D at r: g(r) = sum_q L[q] g(q) (the same values as
// interp_at<D>, so the claims are the same field elements).
template <int D>
__device__ void interp_weights(ef2 r, ef2 (&L)[D + 1]) {
  const u64 inv2 = 0x7FFFFFFF80000001ULL, inv6 = 0xD555555480000001ULL;
  const ef2 r1 = ef_sub(r, ef_from(1)), r2 = ef_sub(r, ef_from(2));
  if (D == 1) {
    L[0] = ef_sub(ef_one(), r);
    L[1] = r;
  } else if (D == 2) {
    L[0] = ef_scale(ef_mul(r1, r2), inv2);
    L[1] = ef_sub(ef_zero(), ef_mul(r, r2));
    L[D] = ef_scale(ef_mul(r, r1), inv2);
  } else {
    const ef2 r3 = ef_sub(r, ef_from(3));
    const ef2 r12 = ef_mul(r1, r2), rr1 = ef_mul(r, r1);
    L[0] = ef_sub(ef_zero(), ef_scale(ef_mul(r12, r3), inv6));
    L[1] = ef_scale(ef_mul(ef_mul(r, r2), r3), inv2);
    L[D - 1] = ef_sub(ef_zero(), ef_scale(ef_mul(rr1, r3), inv2));
    L[D] = ef_scale(ef_mul(rr1, r2), inv6);
  }
}

// Remaining rounds t0..k-1 in one CTA of SC_TAIL_THREADS (NT) threads.  On entry the vectors hold
// `len` entries (len <= TAIL); if `fold`, they hold 2*len entries still to be folded with
// challenge t0 - 1.  The high variable is bound first (pairs i, i + half), so a thread that owns
// the indices congruent to its id modulo NT owns both members of every pair while half >= NT:
//   phase A  rounds with half >= NT: each thread folds its own slice of shared memory, no
//            barrier (at most three rounds: TAIL = 8 NT);
//   hand-over one barrier; warp 0 continues alone;
//   phase B  rounds with 32 <= half < NT: the same with lane l owning l mod 32;
//   phase C  half < 32: one entry per lane, the partner's through a shuffle.
// No round waits for a reduction: each round's sums go to shared memory per warp (phase A) or
// per lane (B, C) and are added up once at the end.  g(1) of every round after the first is
// filled in along the claim chain (see the chain below).
template <int D, bool BIN>
struct TailSmem {
  static constexpr int S = Fac<D, BIN>::S;
  ef2 sv[S][Fac<D, BIN>::TAIL];
  ef2 wsum[3][SC_TAIL_THREADS / 32][D + 1];  // phase A: per-warp sums of its (<= 3) rounds
  ef2 lsum[8][D + 1][32];                     // phases B and C: per-lane sums (<= 7 rounds)
};

template <int D, bool BIN>
__global__ void __launch_bounds__(SC_TAIL_THREADS)
    sc_tail_kernel(Polys<Fac<D, BIN>::S> P, unsigned len, int fold, const ef2* __restrict__ ch,
                   unsigned t0, unsigned k, ef2* __restrict__ rounds_out,
                   ef2* __restrict__ final_out, const ef2* __restrict__ partials,
                   size_t stride, unsigned cap) {
  constexpr int S = Fac<D, BIN>::S;
  constexpr unsigned NT = SC_TAIL_THREADS, NW = NT / 32;
  extern __shared__ __align__(16) unsigned char tail_smem_raw[];
  TailSmem<D, BIN>& sm = *reinterpret_cast<TailSmem<D, BIN>*>(tail_smem_raw);
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // The multi-CTA rounds 0..t0-1: round t's sums over the CTAs that ran it (one warp per round);
  // the claim chain at the end reads them, after the hand-over barrier below.
  for (unsigned t = warp; t < t0; t += NW) {
    const size_t half = (size_t)1 << (k - 1 - t);
    const unsigned nb = (unsigned)min((size_t)cap, (half + SC_THREADS - 1) / SC_THREADS);
    ef2 sr[D + 1];
#pragma unroll
    for (int q = 0; q <= D; ++q) sr[q] = ef_zero();
    const ef2* src = partials + (size_t)t * stride;
    for (unsigned b = lane; b < nb; b += 32)
#pragma unroll
      for (int q = 0; q <= D; ++q) sr[q] = ef_add(sr[q], src[(size_t)b * (D + 1) + q]);
#pragma unroll
    for (int q = 0; q <= D; ++q)
#pragma unroll
      for (int m = 16; m; m >>= 1) sr[q] = ef_add(sr[q], shfl_xor_ef(sr[q], m));
    if (lane == 0)
#pragma unroll
      for (int q = 0; q <= D; ++q) rounds_out[(size_t)t * (D + 1) + q] = sr[q];
  }
  // load, folding with the previous challenge; thread i loads the indices it owns in phase A
  {
    const ef2 r = fold ? ch[t0 - 1] : ef_zero();
    for (unsigned i = threadIdx.x; i < len; i += NT)
#pragma unroll
      for (int j = 0; j < S; ++j)
        sm.sv[j][i] = fold ? ef_lerp(P.p[j][i], P.p[j][i + len], r) : P.p[j][i];
  }
  unsigned L = len, t = t0, ra = 0;
  // phase A
  for (; L >= 2 * NT && t < k; ++t, ++ra, L >>= 1) {
    const unsigned half = L >> 1;
    const ef2 r = ch[t];
    ef2 s[D + 1];
#pragma unroll
    for (int q = 0; q <= D; ++q) s[q] = ef_zero();
    for (unsigned i = threadIdx.x; i < half; i += NT) {
      ef2 lo[S], hi[S];
#pragma unroll
      for (int j = 0; j < S; ++j) lo[j] = sm.sv[j][i], hi[j] = sm.sv[j][i + half];
      add_pair<D, BIN>(lo, hi, s, t > 0);
#pragma unroll
      for (int j = 0; j < S; ++j) sm.sv[j][i] = ef_lerp(lo[j], hi[j], r);
    }
#pragma unroll
    for (int q = 0; q <= D; ++q)
#pragma unroll
      for (int m = 16; m; m >>= 1) s[q] = ef_add(s[q], shfl_xor_ef(s[q], m));
    if (lane == 0)
#pragma unroll
      for (int q = 0; q <= D; ++q) sm.wsum[ra][warp][q] = s[q];
  }
  __syncthreads();  // hand-over: every fold and partial-round sum is visible
  if (warp != 0) return;
  unsigned rb = 0;
  // phase B
  for (; L >= 64 && t < k; ++t, ++rb, L >>= 1) {
    const unsigned half = L >> 1;
    const ef2 r = ch[t];
    ef2 s[D + 1];
#pragma unroll
    for (int q = 0; q <= D; ++q) s[q] = ef_zero();
    for (unsigned i = lane; i < half; i += 32) {
      ef2 lo[S], hi[S];
#pragma unroll
      for (int j = 0; j < S; ++j) lo[j] = sm.sv[j][i], hi[j] = sm.sv[j][i + half];
      add_pair<D, BIN>(lo, hi, s, t > 0);
#pragma unroll
      for (int j = 0; j < S; ++j) sm.sv[j][i] = ef_lerp(lo[j], hi[j], r);
    }
#pragma unroll
    for (int q = 0; q <= D; ++q) sm.lsum[rb][q][lane] = s[q];
  }
  __syncwarp();
  // phase C
  ef2 v[S];
#pragma unroll
  for (int j = 0; j < S; ++j) v[j] = lane < L ? sm.sv[j][lane] : ef_zero();
  for (; L > 1 && t < k; ++t, ++rb, L >>= 1) {
    const unsigned half = L >> 1;
    const ef2 r = ch[t];
    ef2 hi[S];
#pragma unroll
    for (int j = 0; j < S; ++j)
      hi[j] = ef_make(__shfl_down_sync(0xffffffffu, v[j].c0, half),
                      __shfl_down_sync(0xffffffffu, v[j].c1, half));
    ef2 s[D + 1];
#pragma unroll
    for (int q = 0; q <= D; ++q) s[q] = ef_zero();
    if (lane < half) {
      add_pair<D, BIN>(v, hi, s, t > 0);
#pragma unroll
      for (int j = 0; j < S; ++j) v[j] = ef_lerp(v[j], hi[j], r);
    }
#pragma unroll
    for (int q = 0; q <= D; ++q) sm.lsum[rb][q][lane] = s[q];
  }
  __syncwarp();
  // this kernel's round sums (g(1) only for round 0): lane x adds up one (round, q) pair
  const unsigned nra = ra, nrb = rb;
  for (unsigned x = lane; x < (nra + nrb) * (D + 1); x += 32) {
    const unsigned rr = x / (D + 1), q = x % (D + 1);
    const unsigned tt = t0 + rr;
    if (q == 1 && tt > 0) continue;
    ef2 acc = ef_zero();
    if (rr < nra) {
#pragma unroll
      for (unsigned w = 0; w < NW; ++w) acc = ef_add(acc, sm.wsum[rr][w][q]);
    } else {
      for (unsigned l = 0; l < 32; ++l) acc = ef_add(acc, sm.lsum[rr - nra][q][l]);
    }
    rounds_out[(size_t)tt * (D + 1) + q] = acc;
  }
  __threadfence_block();  // the chain below reads these sums from other lanes
  if (lane == 0) {
    if (BIN) {
      final_out[0] = v[0];
      final_out[1] = ef_sub(v[0], ef_one());
#pragma unroll
      for (int j = 1; j < S; ++j) final_out[j + 1] = v[j];
    } else {
#pragma unroll
      for (int j = 0; j < S; ++j) final_out[j] = v[j];
    }
  }
  __syncwarp();
  // The claim chain: g_t(1) = claim_t - g_t(0) for t >= 1, claim_{t+1} = g_t(r_t).  With
  // g_t(r) = sum_q L_q(r) g_t(q), claim_{t+1} = A_t + L_1(r_t) claim_t, A_t collecting the other
  // terms (and A_0 = g_0(r_0), whose g(1) is summed), so lane t prepares its round's A_t and
  // L_1(r_t) in parallel and the claim moves from lane to lane with one product per round.
  ef2 claim = ef_zero();
  for (unsigned c0 = 0; c0 < k; c0 += 32) {
    const unsigned tt = c0 + lane;
    ef2 g[D + 1], L[D + 1], a = ef_zero(), w1 = ef_zero();
    if (tt < k) {
#pragma unroll
      for (int q = 0; q <= D; ++q) g[q] = rounds_out[(size_t)tt * (D + 1) + q];
      interp_weights<D>(ch[tt], L);
#pragma unroll
      for (int q = 0; q <= D; ++q)
        if (q != 1) a = ef_add(a, ef_mul(L[q], g[q]));
      if (tt == 0) {
        a = ef_add(a, ef_mul(L[1], g[1]));
      } else {
        w1 = L[1];
        a = ef_sub(a, ef_mul(L[1], g[0]));
      }
    }
    ef2 mine = ef_zero();  // claim_tt
    for (unsigned j = 0; j < 32 && c0 + j < k; ++j) {
      ef2 next = ef_zero();
      if (lane == j) {
        mine = claim;
        next = ef_add(a, ef_mul(w1, claim));
      }
      claim = ef_make(__shfl_sync(0xffffffffu, next.c0, j), __shfl_sync(0xffffffffu, next.c1, j));
    }
    if (tt < k && tt > 0) rounds_out[(size_t)tt * (D + 1) + 1] = ef_sub(mine, g[0]);
  }
}

template <int D, bool BIN>
void sumcheck_run(ef2* const* polys, unsigned k, const ef2* ch, ef2* rounds_out, ef2* final_out,
                  ef2* partials, cudaStream_t st, unsigned max_blocks) {
  const size_t cap = (max_blocks && max_blocks < SC_MAX_BLOCKS) ? max_blocks : SC_MAX_BLOCKS;
  constexpr int S = Fac<D, BIN>::S;
  Polys<S> P;
  for (int j = 0; j < S; ++j) P.p[j] = polys[j];
  const size_t stride = (size_t)SC_MAX_BLOCKS * (D + 1);
  size_t len = (size_t)1 << k;
  unsigned t = 0;
  int fold = 0;
  while (t < k && len > Fac<D, BIN>::TAIL) {
    if (!(BIN && t == 0) && t + 1 < k && (len >> 1) > Fac<D, BIN>::TAIL) {  // two rounds
      const unsigned nb_t = (unsigned)std::min<size_t>(cap, cdiv(len >> 1, SC_THREADS));
      const unsigned nb_t1 = (unsigned)std::min<size_t>(cap, cdiv(len >> 2, SC_THREADS));
      sc_round2_kernel<D, BIN><<<nb_t1, SC_THREADS, 0, st>>>(
          P, len, fold, fold ? ch + (t - 1) : ch, ch + t, partials + (size_t)t * stride,
          partials + (size_t)(t + 1) * stride, nb_t);
      LGS_LAUNCH_CHECK();
      len >>= 2;
      fold = 1;
      t += 2;
      continue;
    }
    size_t half = len >> 1;
    unsigned blocks = (unsigned)std::min<size_t>(cap, cdiv(half, SC_THREADS));
    if (BIN && t == 0)
      sc_bin_round0_kernel<<<blocks, SC_THREADS, 0, st>>>(P.p[0], P.p[S - 1], half, partials);
    else
      sc_round_kernel<D, BIN><<<blocks, SC_THREADS, 0, st>>>(
          P, half, fold, fold ? ch + (t - 1) : ch, partials + (size_t)t * stride);
    LGS_LAUNCH_CHECK();
    len = half;
    fold = 1;
    ++t;
  }
  tl_mark("sc_passes_end", st);
  // the tail also sums the multi-CTA rounds' partials, and completes their g(1) along the
  // claim chain
  constexpr size_t tail_smem = sizeof(TailSmem<D, BIN>);
  LGS_CUDA(cudaFuncSetAttribute(sc_tail_kernel<D, BIN>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tail_smem));
  sc_tail_kernel<D, BIN><<<1, SC_TAIL_THREADS, tail_smem, st>>>(P, (unsigned)len, fold, ch, t, k,
                                                        rounds_out, final_out, partials, stride,
                                                                 (unsigned)cap);
  LGS_LAUNCH_CHECK();
}
}  // namespace

size_t sumcheck_partials_elems(unsigned k, unsigned d) {
  return (size_t)(k ? k : 1) * SC_MAX_BLOCKS * (d + 1);
}

void sumcheck_prove_dev(ef2* const* polys, unsigned d, unsigned k, const ef2* ch, ef2* rounds_out,
                        ef2* final_out, ef2* partials, cudaStream_t st, unsigned max_blocks) {
  if (k == 0) throw ShapeError("sumcheck: zero variables");
  if (k > 40) throw ShapeError("sumcheck: too many variables");
  switch (d) {
    case 1: sumcheck_run<1, false>(polys, k, ch, rounds_out, final_out, partials, st, max_blocks); break;
    case 2: sumcheck_run<2, false>(polys, k, ch, rounds_out, final_out, partials, st, max_blocks); break;
    case 3: sumcheck_run<3, false>(polys, k, ch, rounds_out, final_out, partials, st, max_blocks); break;
    default: throw ShapeError("sumcheck: 1 to 3 factors supported");
  }
}

void sumcheck_binary_dev(ef2* b, ef2* eq, unsigned k, const ef2* ch, ef2* rounds_out,
                         ef2* final_out, ef2* partials, cudaStream_t st, unsigned max_blocks) {
  if (k == 0 || k > 40) throw ShapeError("sumcheck: variable count out of range");
  ef2* polys[2] = {b, eq};
  sumcheck_run<3, true>(polys, k, ch, rounds_out, final_out, partials, st, max_blocks);
}

}  // namespace lgs
