// Host-side launchers for every device kernel of the prover library.  All of them enqueue on
// the given stream and never synchronize.
#pragma once
#include <algorithm>
#include <cstddef>
#include <vector>

#include "common.cuh"

namespace lgs {

constexpr unsigned SC_MAX_BLOCKS = 296;  // 2 CTAs per SM on a 148-SM B200

// ntt.cu
void build_twiddles(u64* d_tw, cudaStream_t st);
void ntt_batch(const u64* in, size_t in_stride, size_t n_in, u64* out, size_t out_stride,
               unsigned logN, size_t batch, u64* scratch, const u64* tw, cudaStream_t st);
void transpose_u64(const u64* in, u64* out, size_t rows, size_t cols, size_t batch,
                   cudaStream_t st);

// rs_dft.cu: the commitment rows' RS encoding for 2^RS_LOGN_MIN <= N <= 2^RS_LOGN_MAX, from N/2
// (zero-padded) or N input values per row.  z: rows x N scratch.  tables: the context's
// rs_tables_elems() twiddles built by build_rs_tables from the main table.
constexpr unsigned RS_LOGN_MIN = 14, RS_LOGN_MAX = 18;
size_t rs_tables_elems();
size_t rs_table_offset(unsigned logN);
void build_rs_tables(u64* tables, const u64* tw, cudaStream_t st);
bool rs_dft_supported(unsigned logN, size_t n_in);
void rs_dft_rows(const u64* in, size_t ld_in, size_t n_in, u64* out, size_t ld_out,
                 unsigned logN, size_t rows, u64* z, const u64* tables, cudaStream_t st);
// Device-wide rate of the encoding's arithmetic with no memory traffic, per second: op 0 radix-8
// DFTs, op 1 Goldilocks multiplications.  sink: one u64 of device memory.
double rs_alu_rate(int op, unsigned iters, u64* sink, cudaStream_t st);

// hash_tc.cu (tcgen05): also writes the Merkle leaf hashes of H's columns into `leaves`.
void alimb_from_a(const u64* A, uint8_t* alimb, size_t W, cudaStream_t st);
void make_alimb_tmap(const uint8_t* alimb, size_t W, void* tmap_out);
size_t tensor_map_bytes();
void make_i64_tmap(const int64_t* base, size_t rows, size_t inner, unsigned box_rows,
                   void* tmap_out);
// wait_cycles: clock budget of the kernel's bounded waits (0 = the default, about 2 s).
// max_ctas: persistent CTAs (0 = one per SM); fewer leave SMs to concurrent work.
// Rows [row0, row0 + rows) of the codeword only (rows = 0: to the end; both even except at the
// end): H is linear in the rows, so mode 0 writes the rows' partial digest, mode 1 adds it to H,
// and modes 2 and 3 (write, add) also hash the finished H's leaves.
void subset_sum_hash_tc(const void* tmap, const u64* cw, u64* H, u32* leaves, unsigned m,
                        size_t two_n, int* err, cudaStream_t st, uint64_t wait_cycles = 0,
                        unsigned max_ctas = 0, unsigned row0 = 0, unsigned rows = 0,
                        int mode = 2, u64* split_scratch = nullptr);
// When the codeword has fewer 256-column tiles than CTAs, the hash splits its K rows over CTAs
// into this many digest slices (a power of two); split_scratch must then hold splits x 32 x two_n
// values (splits == 1: none needed).
unsigned subset_sum_hash_splits(size_t two_n, unsigned rows, unsigned max_ctas = 0);
// Dense tcgen05 kind::i8 throughput (TOP/s) of back-to-back M128 N256 K32 MMAs on every SM.
double i8_tensor_peak_tops(unsigned iters, int* err, cudaStream_t st);

// merkle.cu
size_t merkle_node_count(size_t nleaves);
size_t merkle_layer_offset(size_t nleaves, unsigned layer);
void merkle_build_from_leaves(u32* nodes, size_t nleaves, cudaStream_t st);
// Up to 16 independent trees (node buffers with their leaf hashes in place) built together:
// one launch per 9 layers of the tallest tree.
void merkle_build_many(u32* const* nodes, const size_t* nleaves, unsigned ntrees, cudaStream_t st);
// Leaf hashes of up to 16 trees in one launch: tree t's leaves are nleaves[t] runs of `words`
// u64 starting at data[t], hashed into nodes[t].
void merkle_leaves_many(const u64* const* data, unsigned words, u32* const* nodes,
                        const size_t* nleaves, unsigned ntrees, cudaStream_t st);
void merkle_leaves_contig(const u64* data, unsigned words, size_t nleaves, u32* nodes,
                          cudaStream_t st);
void gather_u64(const u64* src, const uint64_t* idx, size_t count, unsigned words, u64* dst,
                cudaStream_t st);

// Timeline marks inside multi-kernel helpers (profile level 2, bench.py --mode timeline): an
// event node named "<branch>/<what>" when a prove is being enqueued with timeline marks on this
// host thread, nothing otherwise.
void tl_mark(const char* what, cudaStream_t st);

// sumcheck.cu
size_t sumcheck_partials_elems(unsigned k, unsigned d);
// max_blocks: grid cap of the multi-CTA passes (0 or above SC_MAX_BLOCKS: SC_MAX_BLOCKS).
void sumcheck_prove_dev(ef2* const* polys, unsigned d, unsigned k, const ef2* ch, ef2* rounds_out,
                        ef2* final_out, ef2* partials, cudaStream_t st, unsigned max_blocks = 0);
// The 3-factor sumcheck of [b, b - 1, eq] storing only b and eq (both folded in place).
void sumcheck_binary_dev(ef2* b, ef2* eq, unsigned k, const ef2* ch, ef2* rounds_out,
                         ef2* final_out, ef2* partials, cudaStream_t st, unsigned max_blocks = 0);

// eval.cu
void canon_u64(u64* p, size_t n, cudaStream_t st);  // p[i] = p[i] mod p, in place
struct GatherSeg {
  const u64* src;
  const uint64_t* idx;  // item indices into src (units of `words`)
  uint64_t count;
  uint32_t words;
  u64* dst;
};
void gather_segments(const GatherSeg* segs_dev, unsigned nseg, cudaStream_t st);
void new_eq_dev(const ef2* point, unsigned k, ef2* out, cudaStream_t st);
// MlPoly::fold of the np (1..8) lowest variables: 2^k EF in, 2^(k-np) EF out.
void mle_fold_dev(const ef2* in, unsigned k, const ef2* point, unsigned np, ef2* out,
                  cudaStream_t st);
void combine_eq_dev(const ef2* points, unsigned npts, unsigned k, const ef2* gamma, ef2* out,
                    cudaStream_t st);
size_t eqdot_partials_elems(unsigned k);
// out = sum_i vec[i] * eq_point(i); vec is EF (is_bf = 0) or BF (is_bf = 1).
void eq_dot_dev(const void* vec, int is_bf, const ef2* point, unsigned k, ef2* out,
                ef2* partials, cudaStream_t st);
// The next four read their source address from device memory (`*ref`), so a launch captured in
// a graph reads whichever buffer the slot names when it runs.
void gemv_eq_rows(const u64* const* fref, const ef2* eq, size_t m, size_t n, ef2* out,
                  cudaStream_t st);
void lift_bf(const u64* in, ef2* out, size_t n, u64 minus, cudaStream_t st);
void bits_gather(const u64* const* cwref, size_t two_n, const uint64_t* idx, unsigned s,
                 size_t W, u64* bi, cudaStream_t st);
void g1_build(const u64* const* aref, size_t W, const ef2* eq_a2, unsigned C, ef2* g1,
              cudaStream_t st);
void g2_build(const u64* bi, size_t W, unsigned s, const ef2* eq_r2, ef2* g2, cudaStream_t st);
void v_build(const ef2* eqz1, size_t W, ef2* v, cudaStream_t st);
void y4_dev(const ef2* eq_r2, const ef2* ra, const uint64_t* idx, unsigned s, ef2* out,
            cudaStream_t st);
void sel_build(const uint64_t* idx, const ef2* eq_r2, unsigned s, size_t two_n, ef2* sel,
               cudaStream_t st);
void rs_weights_dev(const ef2* r3, unsigned log2n, size_t n, const u64* tw, ef2* w,
                    cudaStream_t st);
// Basefold batched-open helpers.
struct BfChannelDev {
  const u64* codes;  // leaf-major: D x 2^li elements (1 u64 per BF, 2 per EF)
  const u64* poly;   // full polynomial, BF or EF
  int is_ef;
  unsigned li;
  const ef2* point;  // num_vars = li + R coordinates
};
void bf_combine_dev(const BfChannelDev* chs_dev, unsigned nch, const ef2* coeffs, size_t D,
                    ef2* combined, cudaStream_t st);
void bf_fold_poly_dev(const u64* const* pref, int is_ef, unsigned li, const ef2* point,
                      size_t out_len, ef2* m, cudaStream_t st);
void bf_levels_dev(ef2* levels, size_t D, unsigned R, const ef2* ch, const u64* tw,
                   cudaStream_t st);
// Many MLE evaluations at once: *out = sum_i vec[i] eq_point(i), every vec 2^k EF long.
struct EqDotTask {
  const ef2* vec;
  const ef2* point;
  ef2* out;
};
size_t eq_dot_multi_partials(unsigned k, unsigned ntasks);
void eq_dot_multi_dev(const EqDotTask* tasks_dev, unsigned ntasks, unsigned k, ef2* partials,
                      cudaStream_t st);

}  // namespace lgs
