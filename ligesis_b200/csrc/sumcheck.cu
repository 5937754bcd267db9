// Product sumcheck prover (utils/src/sumcheck.rs:37-84) on the device.
//
// Round t sends g_t(q) = sum_{i < half} prod_j (lo_j + q (hi_j - lo_j)), q = 0..d, with
// lo = P[i], hi = P[i + half] (the HIGH variable is bound first), then folds every factor with
// the round challenge r_t: P[i] = P[i] + r_t (P[i + half] - P[i]).  All challenges come from the
// pre-drawn oracle (utils/src/oracle.rs:10-64), so no round depends on the host: the fold of
// round t-1 is fused into the evaluation pass of round t, large rounds run two at a time in one
// pass (each thread owns four entries, so the in-place fold has no races), and per-CTA partial
// sums go to a scratch array.  Once the vectors are short (1024 entries, 512 for three stored
// factors), one CTA loads them into shared memory, finishes the remaining rounds there, adds up
// the earlier rounds' partials and fills in every round's g(1) along the claim chain.
//
// Binary variant (the B_I check of pcs/src/ligesis.rs:423-428, factors [b, b - 1, eq]): the
// middle factor is always the first minus one (folding is affine), so only b and eq are stored
// and folded; the products, round messages and final evaluations are those of the 3-factor run.
#include "kernels.cuh"

namespace lgs {

namespace {
constexpr unsigned SC_THREADS = 256;

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

// ---- cooperative rounds: G lanes per pair ----------------------------------------------------
// A pair's work is split over a group of G = 4 lanes (8 for three stored factors): lane r < 2S
// loads (and folds with the previous challenge) one of the 2S values lo_j, hi_j, the group
// exchanges them with shuffles, and lane r computes the round polynomial at one point q.  Each
// lane's chain is then one fold and one product (two F_p2 products) instead of all of them:
// used where there are too few pairs to fill the GPU, so a round's time is its chain's latency.
constexpr unsigned SC_COOP_THREADS = 1024;

template <int D, bool BIN>
struct Coop {
  static constexpr int S = Fac<D, BIN>::S;
  static constexpr unsigned G = S <= 2 ? 4 : 8;
};

// The point lane role r evaluates (-1: none): 0..D, or 0, 2, 3 (up to D) once g(1) comes from
// the claim.
template <int D>
__device__ __forceinline__ int coop_q(unsigned r, bool skip1) {
  if (skip1) return r < (unsigned)D ? (r == 0 ? 0 : (int)r + 1) : -1;
  return r <= (unsigned)D ? (int)r : -1;
}

// prod_j (lo_j + q (hi_j - lo_j)), with b (b - 1) for the first factor of the binary check.
template <int D, bool BIN>
__device__ __noinline__ ef2 pair_point(FacVals<Fac<D, BIN>::S> lo, FacVals<Fac<D, BIN>::S> hi,
                                       int q) {
  constexpr int S = Fac<D, BIN>::S;
  ef2 v[S];
#pragma unroll
  for (int j = 0; j < S; ++j) {
    const ef2 d = ef_sub(hi.v[j], lo.v[j]);
    v[j] = lo.v[j];
    for (int c = 0; c < q; ++c) v[j] = ef_add(v[j], d);
  }
  ef2 p = BIN ? ef_mul(v[0], ef_sub(v[0], ef_one())) : v[0];
#pragma unroll
  for (int j = 1; j < S; ++j) p = ef_mul(p, v[j]);
  return p;
}

template <int S>
__device__ __forceinline__ ef2* factor(const Polys<S>& P, unsigned j) {
  ef2* p = P.p[0];
#pragma unroll
  for (int x = 1; x < S; ++x)
    if (j == (unsigned)x) p = P.p[x];
  return p;
}

// Out-of-line F_p2 products for the tail's one-time code (its rounds, the claim chain): the tail
// runs each instruction about once, so instruction fetch, not issue, bounds it, and one shared
// copy of the product is far less code than one inlined copy per use.
__device__ __noinline__ ef2 ef_mul_ol(ef2 a, ef2 b) { return ef_mul(a, b); }
__device__ __noinline__ ef2 ef_lerp_ol(ef2 a, ef2 b, ef2 r) { return ef_lerp(a, b, r); }

__device__ __forceinline__ ef2 shfl_ef(ef2 v, unsigned src) {
  return ef_make(__shfl_sync(0xffffffffu, v.c0, src), __shfl_sync(0xffffffffu, v.c1, src));
}

// One round over `half` pairs, a group of G lanes per pair.  If `fold`, the vectors still hold
// 4 half entries and are folded with *rptr first (results written back to [0, 2 half)); each
// position is read and written by one lane only.  The CTA's sums go to partial[blockIdx.x].
template <int D, bool BIN>
__global__ void __launch_bounds__(SC_COOP_THREADS)
    sc_coop_kernel(Polys<Fac<D, BIN>::S> P, size_t half, int fold, const ef2* __restrict__ rptr,
                   ef2* __restrict__ partial) {
  constexpr int S = Fac<D, BIN>::S;
  constexpr unsigned G = Coop<D, BIN>::G, NWARP = SC_COOP_THREADS / 32;
  __shared__ ef2 red[NWARP][G];
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned r = lane & (G - 1), gb = lane & ~(G - 1);
  const bool skip1 = fold != 0;
  const int q = coop_q<D>(r, skip1);
  const ef2 rp = fold ? *rptr : ef_zero();
  const size_t len = 2 * half, gpb = SC_COOP_THREADS / G;
  const size_t stride = (size_t)gridDim.x * gpb;
  ef2* const mine = factor<S>(P, r >> 1);
  ef2 acc = ef_zero();
  // warp-uniform loop: every lane takes part in the shuffles, idle groups with act = false
  for (size_t w0 = (size_t)blockIdx.x * gpb + warp * (32 / G); w0 < half; w0 += stride) {
    const size_t i = w0 + lane / G;
    const bool act = i < half;
    ef2 val = ef_zero();
    if (act && r < 2 * S) {
      const size_t x = i + (r & 1) * half;
      val = fold ? ef_lerp(mine[x], mine[x + len], rp) : mine[x];
      if (fold) mine[x] = val;
    }
    FacVals<S> lo, hi;
#pragma unroll
    for (int j = 0; j < S; ++j) lo.v[j] = shfl_ef(val, gb + 2 * j), hi.v[j] = shfl_ef(val, gb + 2 * j + 1);
    if (act && q >= 0) acc = ef_add(acc, pair_point<D, BIN>(lo, hi, q));
  }
#pragma unroll
  for (unsigned m = G; m < 32; m <<= 1) acc = ef_add(acc, shfl_xor_ef(acc, m));
  if (lane < G) red[warp][lane] = acc;
  __syncthreads();
  if (threadIdx.x < G) {
    ef2 sum = ef_zero();
#pragma unroll 4
    for (unsigned w = 0; w < NWARP; ++w) sum = ef_add(sum, red[w][threadIdx.x]);
    const int qq = coop_q<D>(threadIdx.x, skip1);
    if (qq >= 0) partial[(size_t)blockIdx.x * (D + 1) + qq] = sum;
    if (skip1 && threadIdx.x == 0) partial[(size_t)blockIdx.x * (D + 1) + 1] = ef_zero();
  }
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

template <int D>
__device__ void interp_weights_ol(ef2 r, ef2 (&L)[D + 1]) {
  const u64 inv2 = 0x7FFFFFFF80000001ULL, inv6 = 0xD555555480000001ULL;
  const ef2 r1 = ef_sub(r, ef_from(1)), r2 = ef_sub(r, ef_from(2));
  if (D == 1) {
    L[0] = ef_sub(ef_one(), r);
    L[1] = r;
  } else if (D == 2) {
    L[0] = ef_scale(ef_mul_ol(r1, r2), inv2);
    L[1] = ef_sub(ef_zero(), ef_mul_ol(r, r2));
    L[D] = ef_scale(ef_mul_ol(r, r1), inv2);
  } else {
    const ef2 r3 = ef_sub(r, ef_from(3));
    const ef2 r12 = ef_mul_ol(r1, r2), rr1 = ef_mul_ol(r, r1);
    L[0] = ef_sub(ef_zero(), ef_scale(ef_mul_ol(r12, r3), inv6));
    L[1] = ef_scale(ef_mul_ol(ef_mul_ol(r, r2), r3), inv2);
    L[D - 1] = ef_sub(ef_zero(), ef_scale(ef_mul_ol(rr1, r3), inv2));
    L[D] = ef_scale(ef_mul_ol(rr1, r2), inv6);
  }
}

// Remaining rounds t0..k-1 in one CTA, with the cooperative pair groups above.  On entry the
// vectors hold `len` entries (len <= TAIL); if `fold`, they hold 2 len entries still to be
// folded with challenge t0 - 1.  The vectors live in shared memory; a round is one group step
// per pair (the fold of round t is written in place by the lane that loaded lo_j, after every
// read of that position) and one barrier.  Each round's sums are reduced within the warp and
// kept per warp; they are added up once after the last round.  g(1) of every round after the
// first is filled in along the claim chain at the end.
constexpr unsigned SC_TAIL_THREADS = SC_COOP_THREADS;
constexpr unsigned SC_TAIL_MAXR = 11;

template <int D, bool BIN>
struct TailSmem {
  static constexpr int S = Fac<D, BIN>::S;
  ef2 sv[S][Fac<D, BIN>::TAIL];
  ef2 red[SC_TAIL_MAXR][SC_TAIL_THREADS / 32][Coop<D, BIN>::G];
};

template <int D, bool BIN>
__global__ void __launch_bounds__(SC_TAIL_THREADS)
    sc_tail_kernel(Polys<Fac<D, BIN>::S> P, unsigned len, int fold, const ef2* __restrict__ ch,
                   unsigned t0, unsigned k, ef2* __restrict__ rounds_out,
                   ef2* __restrict__ final_out, const ef2* __restrict__ partials,
                   size_t stride, unsigned cap) {
  constexpr int S = Fac<D, BIN>::S;
  constexpr unsigned G = Coop<D, BIN>::G, NW = SC_TAIL_THREADS / 32, GPB = SC_TAIL_THREADS / G;
  extern __shared__ __align__(16) unsigned char tail_smem_raw[];
  TailSmem<D, BIN>& sm = *reinterpret_cast<TailSmem<D, BIN>*>(tail_smem_raw);
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned r = lane & (G - 1), gb = lane & ~(G - 1);
  // The multi-CTA rounds 0..t0-1: round t's sums over the CTAs that ran it (one warp per round);
  // the claim chain at the end reads them, after the barriers below.
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
  {
    const ef2 r0 = fold ? ch[t0 - 1] : ef_zero();
    for (unsigned i = threadIdx.x; i < len; i += SC_TAIL_THREADS)
#pragma unroll
      for (int j = 0; j < S; ++j)
        sm.sv[j][i] = fold ? ef_lerp_ol(P.p[j][i], P.p[j][i + len], r0) : P.p[j][i];
  }
  __syncthreads();
  unsigned L = len, t = t0, rr = 0;
  for (; t < k; ++t, ++rr, L >>= 1) {
    const unsigned half = L >> 1;
    const int q = coop_q<D>(r, t > 0);
    const ef2 rt = ch[t];
    ef2 acc = ef_zero();
    for (unsigned w0 = warp * (32 / G); w0 < half; w0 += GPB) {  // warp-uniform
      const unsigned i = w0 + lane / G;
      const bool act = i < half;
      ef2 val = ef_zero();
      if (act && r < 2 * S) val = sm.sv[r >> 1][i + (r & 1) * half];
      FacVals<S> lo, hi;
#pragma unroll
      for (int j = 0; j < S; ++j)
        lo.v[j] = shfl_ef(val, gb + 2 * j), hi.v[j] = shfl_ef(val, gb + 2 * j + 1);
      if (act && q >= 0) acc = ef_add(acc, pair_point<D, BIN>(lo, hi, q));
      if (act && r < 2 * S && (r & 1) == 0) {
        const unsigned j = r >> 1;
        ef2 l = lo.v[0], h = hi.v[0];
#pragma unroll
        for (int x = 1; x < S; ++x)
          if (j == (unsigned)x) l = lo.v[x], h = hi.v[x];
        sm.sv[j][i] = ef_lerp_ol(l, h, rt);
      }
    }
#pragma unroll
    for (unsigned m = G; m < 32; m <<= 1) acc = ef_add(acc, shfl_xor_ef(acc, m));
    if (lane < G) sm.red[rr][warp][lane] = acc;
    __syncthreads();
  }
  // this kernel's round sums (g(1) only for round 0): lane x of warp 0 adds up one (round, role)
  if (warp != 0) return;
  for (unsigned x = lane; x < rr * G; x += 32) {
    const unsigned ro = x / G, role = x % G, tt = t0 + ro;
    const int qq = coop_q<D>(role, tt > 0);
    if (qq < 0) continue;
    ef2 acc = ef_zero();
    for (unsigned w = 0; w < NW; ++w) acc = ef_add(acc, sm.red[ro][w][role]);
    rounds_out[(size_t)tt * (D + 1) + qq] = acc;
  }
  if (lane == 0) {
    if (BIN) {
      final_out[0] = sm.sv[0][0];
      final_out[1] = ef_sub(sm.sv[0][0], ef_one());
#pragma unroll
      for (int j = 1; j < S; ++j) final_out[j + 1] = sm.sv[j][0];
    } else {
#pragma unroll
      for (int j = 0; j < S; ++j) final_out[j] = sm.sv[j][0];
    }
  }
  __threadfence_block();  // the chain below reads these sums from other lanes
  __syncwarp();
  // The claim chain: g_t(1) = claim_t - g_t(0) for t >= 1, claim_{t+1} = g_t(r_t).  With
  // g_t(r) = sum_q L_q(r) g_t(q), claim_{t+1} = A_t + L_1(r_t) claim_t, A_t collecting the other
  // terms (and A_0 = g_0(r_0), whose g(1) is summed): an affine map per round.  Lane t prepares
  // round t's map and an inclusive scan of the compositions (five shuffle steps) gives every
  // lane claim_{t+1}; claim_t is the previous lane's, and the last lane's carries to the next
  // 32 rounds.
  ef2 carry = ef_zero();
  for (unsigned c0 = 0; c0 < k; c0 += 32) {
    const unsigned tt = c0 + lane;
    ef2 g[D + 1], Lw[D + 1], a = ef_zero(), w1 = ef_one();
    if (tt < k) {
#pragma unroll
      for (int qv = 0; qv <= D; ++qv) g[qv] = rounds_out[(size_t)tt * (D + 1) + qv];
      interp_weights_ol<D>(ch[tt], Lw);
      for (int qv = 0; qv <= D; ++qv)
        if (qv != 1) a = ef_add(a, ef_mul_ol(Lw[qv], g[qv]));
      if (tt == 0) {
        a = ef_add(a, ef_mul_ol(Lw[1], g[1]));
        w1 = ef_zero();
      } else {
        w1 = Lw[1];
        a = ef_sub(a, ef_mul_ol(Lw[1], g[0]));
      }
    }
    // inclusive scan: (a, w) after composing lanes c0 .. lane (later maps on the left)
#pragma unroll
    for (unsigned off = 1; off < 32; off <<= 1) {
      const ef2 pa = ef_make(__shfl_up_sync(0xffffffffu, a.c0, off),
                             __shfl_up_sync(0xffffffffu, a.c1, off));
      const ef2 pw = ef_make(__shfl_up_sync(0xffffffffu, w1.c0, off),
                             __shfl_up_sync(0xffffffffu, w1.c1, off));
      if (lane >= off) {
        a = ef_add(a, ef_mul_ol(w1, pa));
        w1 = ef_mul_ol(w1, pw);
      }
    }
    const ef2 incl = ef_add(a, ef_mul_ol(w1, carry));  // claim_{tt + 1}
    ef2 excl = ef_make(__shfl_up_sync(0xffffffffu, incl.c0, 1),
                       __shfl_up_sync(0xffffffffu, incl.c1, 1));
    if (lane == 0) excl = carry;  // claim_tt
    if (tt < k && tt > 0) rounds_out[(size_t)tt * (D + 1) + 1] = ef_sub(excl, g[0]);
    carry = shfl_ef(incl, 31);
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
      sc_coop_kernel<D, BIN><<<blocks, SC_COOP_THREADS, 0, st>>>(
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
