// Eval-path kernels of the LigeSIS prover (pcs/src/ligesis.rs:347-567) and of the Basefold
// shared-domain batched open (pcs/src/basefold.rs:201-218, 648-856): eq tables, eq-weighted
// dot products (MLE evaluations), the a-bar GEMV, the bit-column gather B_I, the sumcheck
// inputs g1/g2/v/sel, RS-link weights, and the batched-FRI channel rounds and codeword folds.
#include "kernels.cuh"

namespace lgs {

namespace {
constexpr unsigned EQ_TILE_LOG = 10;  // eq tables are built per 1024-entry tile

__device__ __forceinline__ ef2 shfl_xor_ef(ef2 v, int m) {
  ef2 r;
  r.c0 = __shfl_xor_sync(0xffffffffu, v.c0, m);
  r.c1 = __shfl_xor_sync(0xffffffffu, v.c1, m);
  return r;
}
// CTA-wide sum of one EF value; valid in every thread afterwards.  red: >= 32 entries.
__device__ ef2 block_sum(ef2 v, ef2* red) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int m = 16; m; m >>= 1) v = ef_add(v, shfl_xor_ef(v, m));
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  ef2 t = lane < nw ? red[lane] : ef_zero();
#pragma unroll
  for (int m = 16; m; m >>= 1) t = ef_add(t, shfl_xor_ef(t, m));
  return t;
}

// tab[j] = prod_{t < b} (bit t of j ? p[t] : 1 - p[t]) for j < 2^b (b <= 10): two direct
// 32-entry half tables (low 5 and high 5 bits) and one product per entry, two barriers.
// Every thread of the CTA must call it; tab is complete when it returns.
__device__ void eq_table_smem(const ef2* p, unsigned b, ef2* tab) {
  __shared__ ef2 half_tabs[64];
  const unsigned b1 = b < 5 ? b : 5, b2 = b - b1;
  const unsigned n1 = 1u << b1, n2 = 1u << b2;
  for (unsigned j = threadIdx.x; j < n1 + n2; j += blockDim.x) {
    const bool hi = j >= n1;
    const unsigned idx = hi ? j - n1 : j, nb = hi ? b2 : b1;
    const ef2* pp = hi ? p + b1 : p;
    ef2 acc = ef_one();
    for (unsigned t = 0; t < nb; ++t)
      acc = ef_mul(acc, ((idx >> t) & 1) ? pp[t] : ef_sub(ef_one(), pp[t]));
    half_tabs[(hi ? 32 : 0) + idx] = acc;
  }
  __syncthreads();
  for (unsigned j = threadIdx.x; j < (1u << b); j += blockDim.x)
    tab[j] = ef_mul(half_tabs[j & (n1 - 1)], half_tabs[32 + (j >> b1)]);
  __syncthreads();
}
// The two half tables of an eq table over p[0 .. b) (b <= 10): lo[j] over the low
// b1 = min(b, 5) variables, hi[j] over the next b2 = b - b1, so that
// eq(p[0 .. b), j) = lo[j mod 2^b1] hi[j >> b1].  Every thread of the CTA must call it; both
// tables are complete when it returns (it ends with a barrier).
__device__ void eq_halves(const ef2* p, unsigned b, ef2* lo, ef2* hi) {
  const unsigned b1 = b < 5 ? b : 5, b2 = b - b1;
  const unsigned n1 = 1u << b1, n2 = 1u << b2;
  for (unsigned j = threadIdx.x; j < n1 + n2; j += blockDim.x) {
    const bool h = j >= n1;
    const unsigned idx = h ? j - n1 : j, nb = h ? b2 : b1;
    const ef2* pp = h ? p + b1 : p;
    ef2 acc = ef_one();
    for (unsigned t = 0; t < nb; ++t)
      acc = ef_mul(acc, ((idx >> t) & 1) ? pp[t] : ef_sub(ef_one(), pp[t]));
    (h ? hi : lo)[idx] = acc;
  }
  __syncthreads();
}
// prod_{t in [b, k)} (bit t of idx ? p[t] : 1 - p[t]), by a whole warp: lane l multiplies the
// terms t = b + l, b + l + 32, and a shuffle tree multiplies the lanes' products (the field
// product does not depend on the order, so every lane gets the same element).  One thread alone
// took a chain of k - b dependent products while the rest of its CTA waited.
__device__ ef2 eq_high_warp(const ef2* p, unsigned b, unsigned k, size_t idx) {
  ef2 acc = ef_one();
  if (k <= b + 6) {  // a short chain: every lane alone, no tree
    for (unsigned t = b; t < k; ++t)
      acc = ef_mul(acc, ((idx >> t) & 1) ? p[t] : ef_sub(ef_one(), p[t]));
    return acc;
  }
  for (unsigned t = b + (threadIdx.x & 31); t < k; t += 32)
    acc = ef_mul(acc, ((idx >> t) & 1) ? p[t] : ef_sub(ef_one(), p[t]));
#pragma unroll
  for (int m = 16; m; m >>= 1) acc = ef_mul(acc, shfl_xor_ef(acc, m));
  return acc;
}
}  // namespace

// ---- gather ------------------------------------------------------------------------------
// GATHER_SPLIT CTAs per segment (blockIdx.y picks a contiguous share of its items), 32-bit index
// math, and eight loads in flight per thread before their stores: a segment of thousands of words
// in one CTA was a long serial chain of dependent loads.
constexpr unsigned GATHER_SPLIT = 8;
__global__ void gather_segments_kernel(const GatherSeg* __restrict__ segs) {
  const GatherSeg s = segs[blockIdx.x];
  const unsigned words = s.words, count = (unsigned)s.count;
  const unsigned per = (count + GATHER_SPLIT - 1) / GATHER_SPLIT;
  const unsigned i0 = min(count, blockIdx.y * per), i1 = min(count, i0 + per);
  const unsigned t_end = i1 * words;
  constexpr unsigned U = 8;
  for (unsigned t0 = i0 * words + threadIdx.x; t0 < t_end; t0 += U * blockDim.x) {
    u64 v[U];
#pragma unroll
    for (unsigned u = 0; u < U; ++u) {
      const unsigned t = t0 + u * blockDim.x;
      if (t < t_end) {
        const unsigned i = t / words, w = t - i * words;
        v[u] = s.src[s.idx[i] * words + w];
      }
    }
#pragma unroll
    for (unsigned u = 0; u < U; ++u) {
      const unsigned t = t0 + u * blockDim.x;
      if (t < t_end) s.dst[t] = v[u];
    }
  }
}
void gather_segments(const GatherSeg* segs_dev, unsigned nseg, cudaStream_t st) {
  if (!nseg) return;
  gather_segments_kernel<<<dim3(nseg, GATHER_SPLIT), 256, 0, st>>>(segs_dev);
  LGS_LAUNCH_CHECK();
}

// ---- eq tables ----------------------------------------------------------------------------
// MlPoly::new_eq (utils/src/poly.rs:44-53): point[0] is the lowest index bit.
// Entry j of a 2^b tile = lo[j mod 2^b1] * H[j >> b1] with H = (the tile's high factor) * hi:
// one F_p2 product per entry.
__global__ void new_eq_kernel(const ef2* __restrict__ point, unsigned k, ef2* __restrict__ out) {
  __shared__ ef2 p[64];
  __shared__ ef2 lo[32], hi[32];
  __shared__ ef2 hfac;
  if (threadIdx.x < k) p[threadIdx.x] = point[threadIdx.x];
  __syncthreads();
  const unsigned b = k < EQ_TILE_LOG ? k : EQ_TILE_LOG;
  const unsigned b1 = b < 5 ? b : 5;
  const size_t base = (size_t)blockIdx.x << b;
  if (threadIdx.x < 32) {
    const ef2 h = eq_high_warp(p, b, k, base);
    if (threadIdx.x == 0) hfac = h;
  }
  eq_halves(p, b, lo, hi);  // ends with a barrier, so hfac is visible
  if (threadIdx.x < (1u << (b - b1))) hi[threadIdx.x] = ef_mul(hi[threadIdx.x], hfac);
  __syncthreads();
  for (unsigned j = threadIdx.x; j < (1u << b); j += blockDim.x)
    out[base + j] = ef_mul(lo[j & ((1u << b1) - 1)], hi[j >> b1]);
}
void new_eq_dev(const ef2* point, unsigned k, ef2* out, cudaStream_t st) {
  if (k > 40) throw ShapeError("new_eq: too many variables");
  unsigned b = k < EQ_TILE_LOG ? k : EQ_TILE_LOG;
  new_eq_kernel<<<(unsigned)((size_t)1 << (k - b)), 256, 0, st>>>(point, k, out);
  LGS_LAUNCH_CHECK();
}

// MlPoly::fold (utils/src/poly.rs:33-42): binds the np lowest variables to point[0 .. np):
// out[i] = sum_{y < 2^np} eq(point, y) in[i 2^np + y], which for np = 1 is the reference's
// s[2i] + (s[2i+1] - s[2i]) r (the same field element).
__global__ void mle_fold_kernel(const ef2* __restrict__ in, size_t nout, unsigned np,
                                const ef2* __restrict__ point, ef2* __restrict__ out) {
  __shared__ ef2 p[8];
  __shared__ ef2 tab[256];
  if (threadIdx.x < np) p[threadIdx.x] = point[threadIdx.x];
  __syncthreads();
  if (np > 1) eq_table_smem(p, np, tab);
  const ef2 r = p[0];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nout;
       i += (size_t)gridDim.x * blockDim.x) {
    const ef2* s = in + (i << np);
    if (np == 1) {
      const ef2 a = s[0], b = s[1];
      out[i] = ef_add(a, ef_mul(r, ef_sub(b, a)));
    } else {
      ef2 acc = ef_mul(tab[0], s[0]);
      for (unsigned y = 1; y < (1u << np); ++y) acc = ef_add(acc, ef_mul(tab[y], s[y]));
      out[i] = acc;
    }
  }
}
void mle_fold_dev(const ef2* in, unsigned k, const ef2* point, unsigned np, ef2* out,
                  cudaStream_t st) {
  if (np < 1 || np > 8 || np > k) throw ShapeError("mle_fold: 1 <= np <= min(8, k)");
  const size_t nout = (size_t)1 << (k - np);
  const unsigned grid = (unsigned)std::min<size_t>(cdiv(nout, 256), 148 * 16);
  mle_fold_kernel<<<grid, 256, 0, st>>>(in, nout, np, point, out);
  LGS_LAUNCH_CHECK();
}

// combine_eq (pcs/src/ligesis.rs:159-171): out = sum_j gamma^j eq_{points[j]}.  Per tile and
// point, gamma^j times the tile's high eq factor is folded into the upper half table, so an
// entry costs one F_p2 product per point.
__global__ void combine_eq_kernel(const ef2* __restrict__ points, unsigned npts, unsigned k,
                                  const ef2* __restrict__ gamma, ef2* __restrict__ out) {
  __shared__ ef2 p[4 * 64];
  __shared__ ef2 lo[4][32], hi[4][32];
  __shared__ ef2 coef[4];
  for (unsigned i = threadIdx.x; i < npts * k; i += blockDim.x) p[i] = points[i];
  __syncthreads();
  const unsigned b = k < EQ_TILE_LOG ? k : EQ_TILE_LOG;
  const unsigned b1 = b < 5 ? b : 5, n2 = 1u << (b - b1);
  const size_t base = (size_t)blockIdx.x << b;
  if (threadIdx.x < 32) {
    ef2 g = ef_one();
    for (unsigned j = 0; j < npts; ++j) {
      const ef2 h = eq_high_warp(p + j * k, b, k, base);
      if (threadIdx.x == 0) coef[j] = ef_mul(g, h);
      g = ef_mul(g, *gamma);
    }
  }
  for (unsigned j = 0; j < npts; ++j) eq_halves(p + j * k, b, lo[j], hi[j]);
  for (unsigned i = threadIdx.x; i < npts * n2; i += blockDim.x)
    hi[i / n2][i % n2] = ef_mul(hi[i / n2][i % n2], coef[i / n2]);
  __syncthreads();
  for (unsigned i = threadIdx.x; i < (1u << b); i += blockDim.x) {
    const unsigned a = i & ((1u << b1) - 1), u = i >> b1;
    ef2 acc = ef_mul(lo[0][a], hi[0][u]);
    for (unsigned j = 1; j < npts; ++j) acc = ef_add(acc, ef_mul(lo[j][a], hi[j][u]));
    out[base + i] = acc;
  }
}
void combine_eq_dev(const ef2* points, unsigned npts, unsigned k, const ef2* gamma, ef2* out,
                    cudaStream_t st) {
  if (npts > 4 || k > 64) throw ShapeError("combine_eq: at most 4 points of 64 variables");
  unsigned b = k < EQ_TILE_LOG ? k : EQ_TILE_LOG;
  combine_eq_kernel<<<(unsigned)((size_t)1 << (k - b)), 256, 0, st>>>(points, npts, k, gamma, out);
  LGS_LAUNCH_CHECK();
}

// ---- eq-weighted dot: MlPoly(vec).eval(point) = sum_i vec[i] eq_point(i) -------------------
template <bool BF>
__global__ void eq_dot_kernel(const void* __restrict__ vec, const ef2* __restrict__ point,
                              unsigned k, ef2* __restrict__ partials) {
  __shared__ ef2 p[64];
  __shared__ ef2 lo[32], hi[32];
  __shared__ ef2 red[32];
  if (threadIdx.x < k) p[threadIdx.x] = point[threadIdx.x];
  __syncthreads();
  const unsigned b = k < EQ_TILE_LOG ? k : EQ_TILE_LOG;
  const unsigned b1 = b < 5 ? b : 5;
  const size_t base = (size_t)blockIdx.x << b;
  eq_halves(p, b, lo, hi);
  ef2 acc = ef_zero();
  if (b1 == 5 && (blockDim.x & 31) == 0) {
    // a thread's entries share their low five bits (blockDim is a multiple of 32):
    // sum_i vec[i] eq(i) = lo[a] * sum_i vec[i] hi[i >> 5], one product per entry
    for (unsigned j = threadIdx.x; j < (1u << b); j += blockDim.x) {
      if (BF) {
        const u64 x = ((const u64*)vec)[base + j];
        acc = ef_add(acc, ef_scale(hi[j >> 5], x));
      } else {
        acc = ef_add(acc, ef_mul(((const ef2*)vec)[base + j], hi[j >> 5]));
      }
    }
    acc = ef_mul(acc, lo[threadIdx.x & 31]);
  } else {
    for (unsigned j = threadIdx.x; j < (1u << b); j += blockDim.x) {
      const ef2 e = ef_mul(lo[j & ((1u << b1) - 1)], hi[j >> b1]);
      if (BF) {
        const u64 x = ((const u64*)vec)[base + j];
        acc = ef_add(acc, ef_scale(e, x));
      } else {
        acc = ef_add(acc, ef_mul(((const ef2*)vec)[base + j], e));
      }
    }
  }
  acc = block_sum(acc, red);
  if (threadIdx.x < 32) {
    const ef2 h = eq_high_warp(p, b, k, base);
    if (threadIdx.x == 0) partials[blockIdx.x] = ef_mul(acc, h);
  }
}
__global__ void sum_partials_kernel(const ef2* __restrict__ partials, size_t n, ef2* out) {
  __shared__ ef2 red[32];
  ef2 acc = ef_zero();
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) acc = ef_add(acc, partials[i]);
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) *out = acc;
}
size_t eqdot_partials_elems(unsigned k) {
  return k > EQ_TILE_LOG ? ((size_t)1 << (k - EQ_TILE_LOG)) : 1;
}
void eq_dot_dev(const void* vec, int is_bf, const ef2* point, unsigned k, ef2* out,
                ef2* partials, cudaStream_t st) {
  if (k > 40) throw ShapeError("eq_dot: too many variables");
  unsigned b = k < EQ_TILE_LOG ? k : EQ_TILE_LOG;
  unsigned grid = (unsigned)((size_t)1 << (k - b));
  if (is_bf)
    eq_dot_kernel<true><<<grid, 256, 0, st>>>(vec, point, k, partials);
  else
    eq_dot_kernel<false><<<grid, 256, 0, st>>>(vec, point, k, partials);
  LGS_LAUNCH_CHECK();
  sum_partials_kernel<<<1, 256, 0, st>>>(partials, grid, out);
  LGS_LAUNCH_CHECK();
}

__global__ void canon_kernel(u64* __restrict__ p, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = gl_canon(p[i]);
}
void canon_u64(u64* p, size_t n, cudaStream_t st) {
  if (!n) return;
  canon_kernel<<<(unsigned)std::min<size_t>(cdiv(n, 256), 148 * 8), 256, 0, st>>>(p, n);
  LGS_LAUNCH_CHECK();
}

// ---- a-bar = eq_{z1}^T F (pcs/src/ligesis.rs:372-379) --------------------------------------
// A CTA owns 64 column pairs (16-byte loads, 512 contiguous bytes per warp and row); its four
// groups of two warps each sum a quarter of the rows, eight rows in flight.  The BF x EF products
// are accumulated unreduced (160-bit sums of 128-bit products) and reduced once per group; the
// groups' field values are added through shared memory.  Four groups give the SM enough warps to
// overlap one group's loads with another's multiply-adds.
constexpr unsigned GEMV_GROUPS = 4;
constexpr unsigned GEMV_PAIRS = 64;  // column pairs per CTA
__global__ void __launch_bounds__(GEMV_GROUPS * GEMV_PAIRS)
    gemv_eq_rows_kernel(const u64* const* __restrict__ fref, const ef2* __restrict__ eq,
                        size_t m, size_t n, ef2* __restrict__ out) {
  __shared__ u64 part[GEMV_GROUPS - 1][GEMV_PAIRS][4];
  const unsigned c = threadIdx.x % GEMV_PAIRS, g = threadIdx.x / GEMV_PAIRS;
  const size_t j = 2 * ((size_t)blockIdx.x * GEMV_PAIRS + c);
  const bool live = j < n;
  const size_t per = (m + GEMV_GROUPS - 1) / GEMV_GROUPS;
  const size_t i0 = min(m, (size_t)g * per), i1 = min(m, i0 + per);
  const u64* __restrict__ f = *fref;
  Acc160 s00, s01, s10, s11;  // column j / j + 1, coordinate c0 / c1
  gl_acc_zero(s00), gl_acc_zero(s01), gl_acc_zero(s10), gl_acc_zero(s11);
  if (live) {
    size_t i = i0;
    for (; i + 8 <= i1; i += 8) {
      ulonglong2 x[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) x[q] = __ldg((const ulonglong2*)(f + (i + q) * n + j));
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const ef2 e = eq[i + q];
        const u64 a = gl_canon(x[q].x), b = gl_canon(x[q].y);
        gl_mac(s00, e.c0, a), gl_mac(s01, e.c1, a), gl_mac(s10, e.c0, b), gl_mac(s11, e.c1, b);
      }
    }
    for (; i < i1; ++i) {
      const ulonglong2 x = __ldg((const ulonglong2*)(f + i * n + j));
      const ef2 e = eq[i];
      const u64 a = gl_canon(x.x), b = gl_canon(x.y);
      gl_mac(s00, e.c0, a), gl_mac(s01, e.c1, a), gl_mac(s10, e.c0, b), gl_mac(s11, e.c1, b);
    }
  }
  u64 r[4] = {gl_acc_reduce(s00), gl_acc_reduce(s01), gl_acc_reduce(s10), gl_acc_reduce(s11)};
  if (g > 0)
#pragma unroll
    for (int t = 0; t < 4; ++t) part[g - 1][c][t] = r[t];
  __syncthreads();
  if (g == 0 && live) {
#pragma unroll
    for (unsigned h = 0; h + 1 < GEMV_GROUPS; ++h)
#pragma unroll
      for (int t = 0; t < 4; ++t) r[t] = gl_add(r[t], part[h][c][t]);
    out[j] = ef_make(r[0], r[1]);
    out[j + 1] = ef_make(r[2], r[3]);
  }
}
void gemv_eq_rows(const u64* const* fref, const ef2* eq, size_t m, size_t n, ef2* out,
                  cudaStream_t st) {
  if (n % 2) throw ShapeError("gemv: n must be even");
  gemv_eq_rows_kernel<<<cdiv(n / 2, GEMV_PAIRS), GEMV_GROUPS * GEMV_PAIRS, 0, st>>>(fref, eq, m,
                                                                                    n, out);
  LGS_LAUNCH_CHECK();
}

// ---- many eq-weighted dots at once: out_t = sum_i vec_t[i] eq_{point_t}(i), all 2^k long ----
__global__ void eq_dot_multi_kernel(const EqDotTask* __restrict__ tasks, unsigned k,
                                    ef2* __restrict__ partials) {
  __shared__ ef2 p[64];
  __shared__ ef2 lo[32], hi[32];
  __shared__ ef2 red[32];
  const EqDotTask task = tasks[blockIdx.y];
  if (threadIdx.x < k) p[threadIdx.x] = task.point[threadIdx.x];
  __syncthreads();
  const unsigned b = k < EQ_TILE_LOG ? k : EQ_TILE_LOG;
  const unsigned b1 = b < 5 ? b : 5;
  const size_t base = (size_t)blockIdx.x << b;
  eq_halves(p, b, lo, hi);
  ef2 acc = ef_zero();
  if (b1 == 5 && (blockDim.x & 31) == 0) {  // one product per entry (see eq_dot_kernel)
    for (unsigned j = threadIdx.x; j < (1u << b); j += blockDim.x)
      acc = ef_add(acc, ef_mul(task.vec[base + j], hi[j >> 5]));
    acc = ef_mul(acc, lo[threadIdx.x & 31]);
  } else {
    for (unsigned j = threadIdx.x; j < (1u << b); j += blockDim.x)
      acc = ef_add(acc, ef_mul(task.vec[base + j],
                               ef_mul(lo[j & ((1u << b1) - 1)], hi[j >> b1])));
  }
  acc = block_sum(acc, red);
  if (threadIdx.x < 32) {
    const ef2 h = eq_high_warp(p, b, k, base);
    if (threadIdx.x == 0) partials[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = ef_mul(acc, h);
  }
}
__global__ void eq_dot_multi_reduce(const EqDotTask* __restrict__ tasks,
                                    const ef2* __restrict__ partials, unsigned ntiles) {
  __shared__ ef2 red[32];
  ef2 acc = ef_zero();
  for (unsigned i = threadIdx.x; i < ntiles; i += blockDim.x)
    acc = ef_add(acc, partials[(size_t)blockIdx.x * ntiles + i]);
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) *tasks[blockIdx.x].out = acc;
}
size_t eq_dot_multi_partials(unsigned k, unsigned ntasks) {
  return (size_t)ntasks * (k > EQ_TILE_LOG ? ((size_t)1 << (k - EQ_TILE_LOG)) : 1);
}
void eq_dot_multi_dev(const EqDotTask* tasks_dev, unsigned ntasks, unsigned k, ef2* partials,
                      cudaStream_t st) {
  if (k > 40 || ntasks == 0 || ntasks > 65535) throw ShapeError("eq_dot_multi: bad sizes");
  const unsigned b = k < EQ_TILE_LOG ? k : EQ_TILE_LOG;
  const unsigned ntiles = (unsigned)((size_t)1 << (k - b));
  eq_dot_multi_kernel<<<dim3(ntiles, ntasks), 256, 0, st>>>(tasks_dev, k, partials);
  LGS_LAUNCH_CHECK();
  eq_dot_multi_reduce<<<ntasks, 256, 0, st>>>(tasks_dev, partials, ntiles);
  LGS_LAUNCH_CHECK();
}

__global__ void lift_bf_kernel(const u64* __restrict__ in, ef2* __restrict__ out, size_t n,
                               u64 minus) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = ef_make(gl_sub(in[i], minus), 0);
}
void lift_bf(const u64* in, ef2* out, size_t n, u64 minus, cudaStream_t st) {
  lift_bf_kernel<<<cdiv(n, 256), 256, 0, st>>>(in, out, n, minus);
  LGS_LAUNCH_CHECK();
}

// ---- B_I: bi[i*s + k] = bit (i % 64) of F'[i / 64][idx[k]] (pcs/src/ligesis.rs:403-410) -----
__global__ void bits_gather_kernel(const u64* const* __restrict__ cwref, size_t two_n,
                                   const uint64_t* __restrict__ idx, unsigned s, size_t rows,
                                   u64* __restrict__ bi) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= rows * s) return;
  const u64* __restrict__ cw = *cwref;
  size_t q = t / s;
  unsigned k = (unsigned)(t % s);
  u64 word = cw[q * two_n + idx[k]];
  for (unsigned b = 0; b < 64; ++b) bi[(q * 64 + b) * s + k] = (word >> b) & 1;
}
void bits_gather(const u64* const* cwref, size_t two_n, const uint64_t* idx, unsigned s,
                 size_t W, u64* bi, cudaStream_t st) {
  size_t rows = W / 64;
  bits_gather_kernel<<<cdiv(rows * s, 128), 128, 0, st>>>(cwref, two_n, idx, s, rows, bi);
  LGS_LAUNCH_CHECK();
}

// g1 = eq_{alpha2}^T A (pcs/src/ligesis.rs:436-444)
__global__ void g1_kernel(const u64* const* __restrict__ aref, size_t W,
                          const ef2* __restrict__ eq, unsigned C, ef2* __restrict__ g1) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W) return;
  const u64* __restrict__ A = *aref;
  ef2 acc = ef_zero();
  for (unsigned r = 0; r < C; ++r) acc = ef_add(acc, ef_scale(eq[r], A[(size_t)r * W + i]));
  g1[i] = acc;
}
void g1_build(const u64* const* aref, size_t W, const ef2* eq_a2, unsigned C, ef2* g1,
              cudaStream_t st) {
  g1_kernel<<<cdiv(W, 256), 256, 0, st>>>(aref, W, eq_a2, C, g1);
  LGS_LAUNCH_CHECK();
}
// g2[i] = sum_k eq_{r2}[k] B[i][idx[k]] (pcs/src/ligesis.rs:445-455); one warp per i.
__global__ void g2_kernel(const u64* __restrict__ bi, size_t W, unsigned s,
                          const ef2* __restrict__ eq, ef2* __restrict__ g2) {
  size_t i = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31;
  if (i >= W) return;
  ef2 acc = ef_zero();
  for (unsigned k = lane; k < s; k += 32)
    if (bi[i * s + k]) acc = ef_add(acc, eq[k]);
#pragma unroll
  for (int m = 16; m; m >>= 1) acc = ef_add(acc, shfl_xor_ef(acc, m));
  if (lane == 0) g2[i] = acc;
}
void g2_build(const u64* bi, size_t W, unsigned s, const ef2* eq_r2, ef2* g2, cudaStream_t st) {
  g2_kernel<<<cdiv(W * 32, 256), 256, 0, st>>>(bi, W, s, eq_r2, g2);
  LGS_LAUNCH_CHECK();
}
// v[i] = eq_{z1}[i / 64] * 2^(i % 64) (pcs/src/ligesis.rs:474-476)
__global__ void v_kernel(const ef2* __restrict__ eqz1, size_t W, ef2* __restrict__ v) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W) return;
  ef2 e = eqz1[i / 64];
  unsigned sh = (unsigned)(i % 64);
  v[i] = ef_make(gl_shl(e.c0, sh), gl_shl(e.c1, sh));
}
void v_build(const ef2* eqz1, size_t W, ef2* v, cudaStream_t st) {
  v_kernel<<<cdiv(W, 256), 256, 0, st>>>(eqz1, W, v);
  LGS_LAUNCH_CHECK();
}
// y4 = sum_k eq_{r2}[k] RS(a)[idx[k]] (pcs/src/ligesis.rs:458)
__global__ void y4_kernel(const ef2* __restrict__ eq, const ef2* __restrict__ ra,
                          const uint64_t* __restrict__ idx, unsigned s, ef2* out) {
  __shared__ ef2 red[32];
  ef2 acc = ef_zero();
  for (unsigned k = threadIdx.x; k < s; k += blockDim.x) acc = ef_add(acc, ef_mul(eq[k], ra[idx[k]]));
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) *out = acc;
}
void y4_dev(const ef2* eq_r2, const ef2* ra, const uint64_t* idx, unsigned s, ef2* out,
            cudaStream_t st) {
  y4_kernel<<<1, 128, 0, st>>>(eq_r2, ra, idx, s, out);
  LGS_LAUNCH_CHECK();
}
__global__ void sel_scatter_kernel(const uint64_t* __restrict__ idx, const ef2* __restrict__ eq,
                                   unsigned s, ef2* __restrict__ sel) {
  unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < s) sel[idx[k]] = eq[k];
}
void sel_build(const uint64_t* idx, const ef2* eq_r2, unsigned s, size_t two_n, ef2* sel,
               cudaStream_t st) {
  LGS_CUDA(cudaMemsetAsync(sel, 0, two_n * sizeof(ef2), st));
  sel_scatter_kernel<<<cdiv(s, 128), 128, 0, st>>>(idx, eq_r2, s, sel);
  LGS_LAUNCH_CHECK();
}
// w[k] = prod_t (1 - r3[t] + r3[t] g^((2^t k) mod 2n)) (pcs/src/ligesis.rs:553-567)
__global__ void rs_weights_kernel(const ef2* __restrict__ r3, unsigned log2n, size_t n,
                                  const u64* __restrict__ tw, ef2* __restrict__ w) {
  __shared__ ef2 r[64];
  if (threadIdx.x < log2n) r[threadIdx.x] = r3[threadIdx.x];
  __syncthreads();
  size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const size_t mask = ((size_t)2 << (log2n - 1)) - 1;
  const unsigned shift = TW_LOG - log2n;
  ef2 prod = ef_one();
  for (unsigned t = 0; t < log2n; ++t) {
    size_t e = (k << t) & mask;
    u64 gp = __ldg(tw + (e << shift));
    ef2 term = ef_add(ef_sub(ef_one(), r[t]), ef_scale(r[t], gp));
    prod = ef_mul(prod, term);
  }
  w[k] = prod;
}
void rs_weights_dev(const ef2* r3, unsigned log2n, size_t n, const u64* tw, ef2* w,
                    cudaStream_t st) {
  if (log2n > TW_LOG || log2n > 64) throw ShapeError("rs_weights: domain too large");
  rs_weights_kernel<<<cdiv(n, 256), 256, 0, st>>>(r3, log2n, n, tw, w);
  LGS_LAUNCH_CHECK();
}

// ---- Basefold batched open ------------------------------------------------------------------
// Level-0 combined codeword (pcs/src/basefold.rs:660-666, 735-741):
// combined[i] = sum_ch coeffs[ch] sum_j eq4_ch[j] codes_ch[i][j].
__global__ void bf_combine_kernel(const BfChannelDev* __restrict__ chs, unsigned nch,
                                  const ef2* __restrict__ coeffs, size_t D,
                                  ef2* __restrict__ combined) {
  __shared__ ef2 wts[4][64];
  __shared__ ef2 pts[4][8];
  for (unsigned c = 0; c < nch; ++c) {
    if (threadIdx.x < chs[c].li) pts[c][threadIdx.x] = chs[c].point[threadIdx.x];
  }
  __syncthreads();
  for (unsigned c = 0; c < nch; ++c) {
    eq_table_smem(pts[c], chs[c].li, wts[c]);
    for (unsigned j = threadIdx.x; j < (1u << chs[c].li); j += blockDim.x)
      wts[c][j] = ef_mul(wts[c][j], coeffs[c]);
    __syncthreads();
  }
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D) return;
  ef2 acc = ef_zero();
  for (unsigned c = 0; c < nch; ++c) {
    const unsigned L = 1u << chs[c].li;
    if (chs[c].is_ef) {
      const ef2* row = (const ef2*)chs[c].codes + i * L;
      for (unsigned j = 0; j < L; ++j) acc = ef_add(acc, ef_mul(wts[c][j], row[j]));
    } else {
      const u64* row = chs[c].codes + i * L;
      for (unsigned j = 0; j < L; ++j) acc = ef_add(acc, ef_scale(wts[c][j], row[j]));
    }
  }
  combined[i] = acc;
}
void bf_combine_dev(const BfChannelDev* chs_dev, unsigned nch, const ef2* coeffs, size_t D,
                    ef2* combined, cudaStream_t st) {
  if (nch > 4) throw ShapeError("basefold: at most 4 channels per launch");
  bf_combine_kernel<<<cdiv(D, 256), 256, 0, st>>>(chs_dev, nch, coeffs, D, combined);
  LGS_LAUNCH_CHECK();
}

// m = poly.fold(point[0..li]) (pcs/src/basefold.rs:667-668): m[t] = sum_j eq4[j] poly[t 2^li + j].
__global__ void bf_fold_poly_kernel(const u64* const* __restrict__ pref, int is_ef, unsigned li,
                                    const ef2* __restrict__ point, size_t out_len,
                                    ef2* __restrict__ m) {
  __shared__ ef2 pts[8];
  __shared__ ef2 wts[64];
  if (threadIdx.x < li) pts[threadIdx.x] = point[threadIdx.x];
  __syncthreads();
  eq_table_smem(pts, li, wts);
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= out_len) return;
  const u64* __restrict__ poly = *pref;
  const unsigned L = 1u << li;
  ef2 acc = ef_zero();
  if (is_ef) {
    const ef2* row = (const ef2*)poly + t * L;
    for (unsigned j = 0; j < L; ++j) acc = ef_add(acc, ef_mul(wts[j], row[j]));
  } else {
    const u64* row = poly + t * L;
    for (unsigned j = 0; j < L; ++j) acc = ef_add(acc, ef_scale(wts[j], row[j]));
  }
  m[t] = acc;
}
void bf_fold_poly_dev(const u64* const* pref, int is_ef, unsigned li, const ef2* point,
                      size_t out_len, ef2* m, cudaStream_t st) {
  if (li > 6) throw ShapeError("basefold: log_interleave above 6");
  bf_fold_poly_kernel<<<cdiv(out_len, 256), 256, 0, st>>>(pref, is_ef, li, point, out_len, m);
  LGS_LAUNCH_CHECK();
}

// The R codeword folds of the batched open (eq_fold_codeword, pcs/src/basefold.rs:201-218):
// level t+1[i] = (1 - r_t)(x + nx)/2 + r_t (x - nx) g_len^(-i) / 2, x = level t[i],
// nx = level t[i + len/2].  Level k (length D >> k) is stored at offset D (2 - 2^(1-k)).
// Levels longer than BF_TAIL are folded by one grid-wide launch each; the rest of the chain
// (at most 2 BF_TAIL values) is finished by one CTA in shared memory.
constexpr unsigned BF_TAIL = 2048;

__device__ __forceinline__ ef2 bf_fold_pair(ef2 x, ef2 nx, ef2 r, size_t i, size_t len,
                                            const u64* __restrict__ tw) {
  const u64 inv2 = 0x7FFFFFFF80000001ULL;  // (p + 1) / 2
  const unsigned lg = 63 - __clzll((long long)len);
  const u64 ginv = i ? __ldg(tw + ((len - i) << (TW_LOG - lg))) : 1;
  const ef2 pe = ef_scale(ef_add(x, nx), inv2);
  const ef2 po = ef_scale(ef_scale(ef_sub(x, nx), ginv), inv2);
  return ef_add(pe, ef_mul(r, ef_sub(po, pe)));
}

__global__ void __launch_bounds__(256)
    bf_level_kernel(ef2* __restrict__ levels, size_t off, size_t len, const ef2* __restrict__ ch,
                    unsigned t, const u64* __restrict__ tw) {
  const size_t h = len >> 1, i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= h) return;
  levels[off + len + i] = bf_fold_pair(levels[off + i], levels[off + i + h], ch[t], i, len, tw);
}

__global__ void __launch_bounds__(1024)
    bf_levels_tail_kernel(ef2* __restrict__ levels, size_t off, unsigned len, unsigned t0,
                          unsigned R, const ef2* __restrict__ ch, const u64* __restrict__ tw) {
  extern __shared__ ef2 sl[];  // the chain from level t0 on: < 2 len values
  for (unsigned i = threadIdx.x; i < len; i += blockDim.x) sl[i] = levels[off + i];
  __syncthreads();
  unsigned cur = 0;
  for (unsigned t = t0; t < R; ++t) {
    const ef2 r = ch[t];
    const unsigned h = len >> 1;
    for (unsigned i = threadIdx.x; i < h; i += blockDim.x) {
      const ef2 v = bf_fold_pair(sl[cur + i], sl[cur + i + h], r, i, len, tw);
      sl[cur + len + i] = v;
      levels[off + cur + len + i] = v;
    }
    __syncthreads();
    cur += len;
    len = h;
  }
}

void bf_levels_dev(ef2* levels, size_t D, unsigned R, const ef2* ch, const u64* tw,
                   cudaStream_t st) {
  if (R < 1 || R > 30) throw ShapeError("basefold: unsupported round count");
  size_t off = 0, len = D;
  unsigned t = 0;
  for (; t < R && len > BF_TAIL; ++t) {
    bf_level_kernel<<<cdiv(len / 2, 256), 256, 0, st>>>(levels, off, len, ch, t, tw);
    LGS_LAUNCH_CHECK();
    off += len;
    len >>= 1;
  }
  if (t < R) {
    const size_t smem = 2 * len * sizeof(ef2);
    LGS_CUDA(cudaFuncSetAttribute(bf_levels_tail_kernel,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    bf_levels_tail_kernel<<<1, 1024, smem, st>>>(levels, off, (unsigned)len, t, R, ch, tw);
    LGS_LAUNCH_CHECK();
  }
}

}  // namespace lgs
