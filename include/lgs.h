/* LigeSIS / Basefold prover for B200 (sm_100a) — the C ABI of liblgs.so.
 *
 * Each entry point stands in for a function of the reference Rust crate paulguoyanpei/ligesis
 * (paths are inside that project).  Plain pointers and sizes only: BF (Goldilocks) values are
 * uint64_t (reduced mod p = 2^64 - 2^32 + 1 on input), EF (BinomialExtensionField<BF,2>) values
 * are two consecutive uint64_t (c0, c1).  Nothing throws across this boundary: every call
 * returns an lgs_status, and lgs_last_error() describes the last failure on the calling thread.
 * A context owns one CUDA stream on one device; use one context per host thread.
 */
#ifndef LGS_H
#define LGS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LGS_OK = 0,
  LGS_ERR_BAD_SHAPE = 1,        /* setup's shared-domain precondition, or an unsupported size */
  LGS_ERR_OOM = 2,              /* device allocation failed */
  LGS_ERR_ORACLE_EXHAUSTED = 3, /* the randomness oracle has too few fields/ints left */
  LGS_ERR_DEVICE_TIMEOUT = 4,   /* a bounded device wait gave up */
  LGS_ERR_BAD_ARG = 5,          /* null pointer, wrong length, mismatched key/commitment */
  LGS_ERR_CUDA = 6,             /* any other CUDA error */
  LGS_ERR_INTERNAL = 7,
  LGS_ERR_BUFFER_TOO_SMALL = 8  /* *len holds the size needed */
} lgs_status;

typedef struct lgs_ctx lgs_ctx;
typedef struct lgs_pk lgs_pk;                   /* ProvingKey (pcs/src/ligesis.rs:67-74) */
typedef struct lgs_commit_data lgs_commit_data; /* CommitData (pcs/src/ligesis.rs:88-97) */

const char* lgs_last_error(void);
const char* lgs_version(void);

/* Context: device, stream, twiddle table, scratch arena.  `flags` is reserved (pass 0). */
lgs_status lgs_ctx_create(int device, unsigned flags, lgs_ctx** out);
void lgs_ctx_destroy(lgs_ctx* ctx);
/* The cudaStream_t every call of this context enqueues on (for event timing). */
lgs_status lgs_ctx_stream(lgs_ctx* ctx, void** stream);

/* Ligesis::setup (pcs/src/ligesis.rs:239-273).  A: the 32 x (64 * 2^log_m) subset-sum matrix,
 * row-major (SubsetSumHash::new, pcs/src/subset_sum.rs:31-39, sampled by the caller).
 * com_a receives the Basefold commitment to the flattened A. */
lgs_status lgs_setup(lgs_ctx* ctx, unsigned log_m, unsigned log_n, const uint64_t* A,
                     lgs_pk** pk, uint8_t com_a[32]);
/* A key for Ligesis::commit alone (pcs/src/ligesis.rs:277-325, whose RS encoding, hash and
 * Merkle tree take any m x n): the reference's setup (:239-273) asserts the shared-domain window
 * log_m + 7 <= log_n <= log_m + 17 that only the prove needs, so square shapes such as
 * 2^12 x 2^12 can be committed only through this key.  It holds A and its limbs, no Basefold
 * commitment of A; lgs_prove rejects it (LGS_ERR_BAD_SHAPE).  Needs log_m <= 13, 7 <= log_n. */
lgs_status lgs_setup_commit_only(lgs_ctx* ctx, unsigned log_m, unsigned log_n, const uint64_t* A,
                                 lgs_pk** pk);
void lgs_pk_free(lgs_pk* pk);

/* Ligesis::commit (pcs/src/ligesis.rs:277-325).  f: 2^(log_m+log_n) BF evaluations in host
 * memory (MlPoly<BF>, utils/src/poly.rs:4).  root receives the LigesisCommit. */
lgs_status lgs_commit(lgs_ctx* ctx, const lgs_pk* pk, const uint64_t* f, size_t len,
                      uint8_t root[32], lgs_commit_data** out);
/* Same, with f already in device memory of the context's device. */
lgs_status lgs_commit_device(lgs_ctx* ctx, const lgs_pk* pk, const uint64_t* f_dev, size_t len,
                             uint8_t root[32], lgs_commit_data** out);
/* Ligesis::commit without waiting for the device: the work is enqueued on the context's stream
 * and *out is at once usable by lgs_prove on the same context (stream order), so the prove's
 * host-side planning overlaps the commit's device work.  f is host memory (f_on_device = 0; read
 * before the call returns) or device memory of the context's device (f_on_device = 1; copied,
 * must stay unchanged until the commit is done; f_on_device = 2: lent, not copied: the
 * commitment reads the caller's buffer until lgs_commit_data_free, so it must stay allocated
 * and unchanged until then, as the reference's commit owns f).  lgs_commit_root waits for the
 * commit and returns the
 * LigesisCommit root (and reports a failed bounded device wait).  The same computation as
 * lgs_commit, so the root and every later proof are identical. */
lgs_status lgs_commit_async(lgs_ctx* ctx, const lgs_pk* pk, const uint64_t* f, size_t len,
                            int f_on_device, lgs_commit_data** out);
lgs_status lgs_commit_root(lgs_ctx* ctx, lgs_commit_data* cd, uint8_t root[32]);
void lgs_commit_data_free(lgs_commit_data* cd);
/* Copy a commitment intermediate to host memory: which = 0 the RS codeword F' (m x 2n),
 * 1 the digest H (32 x 2n).  count must equal the element count. */
lgs_status lgs_commit_read(lgs_ctx* ctx, const lgs_commit_data* cd, int which, uint64_t* out,
                           size_t count);

/* Oracle draws one prove/verify consumes (RandomOracle cursors, utils/src/oracle.rs:94-116). */
lgs_status lgs_oracle_need(unsigned log_m, unsigned log_n, size_t* fields, size_t* ints);

/* Ligesis::prove (pcs/src/ligesis.rs:347-549).  z: log_m + log_n EF (z2 = the low log_n).
 * fields/ints: the RandomOracle arrays (EF and u64); cursors[0..2] = (fields, ints) positions,
 * advanced on success.  *proof points at the encoded LigesisProof (layout in proof.hpp),
 * owned by the context and valid until its next lgs_prove. */
lgs_status lgs_prove(lgs_ctx* ctx, const lgs_pk* pk, const lgs_commit_data* cd,
                     const uint64_t* z, size_t zlen, const uint64_t* fields, size_t nfields,
                     const uint64_t* ints, size_t nints, uint64_t cursors[2],
                     const uint8_t** proof, size_t* proof_len);

/* Ligesis::verify (pcs/src/ligesis.rs:569-756), on the host.  *accept = 1 or 0. */
lgs_status lgs_verify(unsigned log_m, unsigned log_n, const uint8_t com_a[32],
                      const uint8_t root[32], const uint64_t* z, size_t zlen,
                      const uint8_t* proof, size_t proof_len, const uint64_t* fields,
                      size_t nfields, const uint64_t* ints, size_t nints, uint64_t cursors[2],
                      int* accept);

/* ---- standalone Basefold PCS (pcs/src/basefold.rs) ----
 * Basefold::commit_{base,ext}_on_domain (:341-382; commit_base/commit_ext are log_interleave 6,
 * :309-339): poly holds 2^n values, BF (is_ef = 0, one u64 each) or EF (is_ef = 1, c0 c1),
 * split into 2^log_interleave interleaved chunks (MlPoly::split), each RS-encoded at rate
 * 2^-code_rate; root receives the BasefoldCommit.  The handle keeps the prover state
 * (BasefoldProverState, :46-58) on the device until lgs_basefold_free.
 * Limits: 1 <= log_interleave + 1 <= n, log_interleave <= 6, n - log_interleave + code_rate
 * <= 22. */
typedef struct lgs_basefold lgs_basefold;
lgs_status lgs_basefold_commit(lgs_ctx* ctx, const uint64_t* poly, size_t len, int is_ef,
                               unsigned code_rate, unsigned log_interleave, uint8_t root[32],
                               lgs_basefold** out);
void lgs_basefold_free(lgs_basefold* b);
/* Basefold::prove (:384-516) at an n-coordinate EF point; the RandomOracle arrays and cursors as
 * for lgs_prove (it draws n - log_interleave fields, then ceil(100 / code_rate) ints).  *proof is
 * the encoded BasefoldProof ("LGSB", proof.hpp), owned by the context until its next prove. */
lgs_status lgs_basefold_prove(lgs_ctx* ctx, const lgs_basefold* b, const uint64_t* point,
                              size_t plen, const uint64_t* fields, size_t nfields,
                              const uint64_t* ints, size_t nints, uint64_t cursors[2],
                              const uint8_t** proof, size_t* proof_len);
/* Basefold::verify (:518-642), on the host.  *accept = 1 or 0. */
lgs_status lgs_basefold_verify(const uint8_t root[32], const uint64_t* point, size_t plen,
                               const uint8_t* proof, size_t proof_len, const uint64_t* fields,
                               size_t nfields, const uint64_t* ints, size_t nints,
                               uint64_t cursors[2], int* accept);

/* ---- GKR fraction sum and GKR-LogUp lookup (logup/src/frac_sum.rs, logup/src/lookup.rs) ----
 * EF arrays hold 2 u64 per value (c0, c1), canonical.  With on_device = 1 the input pointers are
 * device pointers on the context's device (16-byte aligned) and are only read; otherwise host
 * memory.  `cursor` is the RandomOracle's fields cursor (in/out); these provers draw no ints.
 * Proofs are owned by the context until its next prove.
 *
 * frac_sum::prove (:110-161): proves sum_i p_i / q_i = num / den over n = 2^k fractions (p NULL:
 * every numerator is one), drawing k (k + 3) / 2 fields.  point receives the reduced input point
 * (k EF, low-bit-first) and claim p_in(point), q_in(point) (2 EF).  The proof is "LGSF"
 * (num, den, then per layer r its r round polynomials g(0..3) and the leaves A0 A1 B0 B1).
 * Limit: k <= 28. */
lgs_status lgs_frac_sum_prove(lgs_ctx* ctx, const uint64_t* p, const uint64_t* q, size_t n,
                              int on_device, const uint64_t* fields, size_t nfields,
                              uint64_t* cursor, const uint8_t** proof, size_t* proof_len,
                              uint64_t* point, uint64_t claim[4]);
/* frac_sum::verify (:221-258), on the host: *accept = 1 with point (point_cap EF at most) and
 * claim filled, or 0 (the reference's None). */
lgs_status lgs_frac_sum_verify(const uint8_t* proof, size_t proof_len, const uint64_t* fields,
                               size_t nfields, uint64_t* cursor, uint64_t* point,
                               size_t point_cap, uint64_t claim[4], int* accept);
/* lookup::prove_with_opening_points (lookup.rs:119-143): every query a_i (m = 2^mu) lies in the
 * table t (n = 2^nu distinct values) with multiplicities e (n values).  Draws alpha, then the
 * query circuit's and the table circuit's fields.  zq / zt receive the opening points (mu / nu
 * EF).  The proof is "LGSL" followed by the two "LGSF" proofs. */
lgs_status lgs_lookup_prove(lgs_ctx* ctx, const uint64_t* a, size_t m, const uint64_t* t,
                            const uint64_t* e, size_t n, int on_device, const uint64_t* fields,
                            size_t nfields, uint64_t* cursor, const uint8_t** proof,
                            size_t* proof_len, uint64_t* zq, uint64_t* zt);
/* lookup::verify (:191-229), on the host: *accept = 1 with the opening claims a(zq), e(zt), t(zt)
 * in vals (3 EF) and the points in zq / zt, or 0. */
lgs_status lgs_lookup_verify(const uint8_t* proof, size_t proof_len, const uint64_t* fields,
                             size_t nfields, uint64_t* cursor, uint64_t* zq, size_t zq_cap,
                             uint64_t* zt, size_t zt_cap, uint64_t vals[6], int* accept);

/* ---- proofsys' integer witness (proofsys/src/tensor.rs, proofsys/src/model.rs) ----
 * The rescaled linear layer of the integer GPT-2 (model.rs:360-361): Q, REM =
 * floor_div_const_with_rem(X.matmul(W), divisor) (tensor.rs:76-89, :121-133) and Y = Q + bias
 * (add_row_vector, :51-60); with w_transposed, X.matmul_transposed_rhs(W) (:91-104) and W is
 * cols x inner.  X is rows x inner, all row-major int64; REM lies in [0, divisor); bias (cols) and
 * y_field (rows x cols, encode_i64(Y) as canonical Goldilocks, witness.rs:102-108) may be NULL.
 * on_device = 1: every array is a device pointer on the context's device.  A product or a Q + bias
 * outside the int64 range (where the reference panics) gives LGS_ERR_BAD_SHAPE. */
lgs_status lgs_linear_witness(lgs_ctx* ctx, const int64_t* x, size_t rows, size_t inner,
                              const int64_t* w, size_t cols, int w_transposed,
                              const int64_t* bias, int64_t divisor, int on_device, int64_t* q,
                              int64_t* rem, int64_t* y, uint64_t* y_field);
/* layer_norm of the integer GPT-2 (model.rs:241-279): for each of `rows` rows of X (d columns),
 * sum_x, sum_x2, var_sum = d sum_x2 - sum_x^2 and std = round_sqrt(var_sum + 1) (tensor.rs:
 * 218-222); for each entry dividend = gain (d x - sum_x), quotient = floor(dividend / std),
 * output = quotient + bias.  Per-row outputs hold rows values, per-entry ones rows x d.  A sum or
 * a dividend outside the int64 range gives LGS_ERR_BAD_SHAPE. */
lgs_status lgs_layer_norm_witness(lgs_ctx* ctx, const int64_t* x, size_t rows, size_t d,
                                  const int64_t* gain, const int64_t* bias, int on_device,
                                  int64_t* sum_x, int64_t* sum_x2, int64_t* var_sum,
                                  int64_t* stdv, int64_t* dividend, int64_t* quotient,
                                  int64_t* output);
/* softmax of the integer GPT-2 attention (model.rs:409-443), causal, for `heads` score matrices
 * of n x n (heads x n x n, row-major): x_max[h][i] = max_{j <= i} s, exp[h][i][j] =
 * exp_lut[s - x_max + offset] and prob[h][i][j] = floor(exp scale / sum_exp) for j <= i (zero
 * above the diagonal), sum_exp[h][i] = sum_j exp.  An index outside the table or a zero sum gives
 * LGS_ERR_BAD_SHAPE (the reference asserts). */
lgs_status lgs_softmax_witness(lgs_ctx* ctx, const int64_t* scores, unsigned heads, unsigned n,
                               const int64_t* exp_lut, size_t lut_len, int64_t offset,
                               int64_t scale, int on_device, int64_t* x_max, int64_t* exp,
                               int64_t* sum_exp, int64_t* prob);
/* out[i] = lut[v[i] + offset], the GELU activation of the MLP (model.rs:362-373); an index
 * outside the table gives LGS_ERR_BAD_SHAPE. */
lgs_status lgs_lut_gather(lgs_ctx* ctx, const int64_t* v, size_t count, const int64_t* lut,
                          size_t lut_len, int64_t offset, int on_device, int64_t* out);

/* ---- batched and served proving (the reference proves one polynomial at a time on one
 * thread, pcs/benches/ligesis.rs:20-60) ----
 * An engine owns `lanes` contexts on one device, each driven by its own host thread, so the
 * commits and proofs of many jobs of uneven sizes run on the GPU together.  A queued job starts
 * when a lane is free and its device-memory estimate fits the HBM budget (FIFO).  Every job runs
 * the same lgs_commit + lgs_prove computation, so its root and proof are byte-identical to the
 * one-at-a-time path.  The job's host buffers and its proving key must stay alive and unchanged
 * until the job has been waited for. */
typedef struct lgs_engine lgs_engine;
typedef struct {
  const lgs_pk* pk;
  const uint64_t* f; /* host, 2^(log_m+log_n) BF */
  size_t len;
  const uint64_t* z; /* log_m + log_n EF */
  size_t zlen;
  const uint64_t* fields; /* RandomOracle arrays and the cursors this proof starts at */
  size_t nfields;
  const uint64_t* ints;
  size_t nints;
  uint64_t cursors[2];
} lgs_job;
typedef struct {
  lgs_status status;
  uint8_t root[32];
  uint8_t* proof; /* owned by the caller after lgs_engine_wait: lgs_engine_free_proof */
  size_t proof_len;
  uint64_t cursors[2]; /* advanced cursors */
  double submit_ms, start_ms, done_ms; /* engine clock (ms since lgs_engine_create) */
} lgs_result;
/* hbm_budget 0: 90% of the device memory free at creation. */
lgs_status lgs_engine_create(int device, unsigned lanes, size_t hbm_budget, lgs_engine** out);
void lgs_engine_destroy(lgs_engine* e);
lgs_status lgs_engine_submit(lgs_engine* e, const lgs_job* job, uint64_t* ticket);
/* Blocks until the job is done (timeout_ms < 0: no limit); the ticket is then released. */
lgs_status lgs_engine_wait(lgs_engine* e, uint64_t ticket, double timeout_ms, lgs_result* out);
void lgs_engine_free_proof(uint8_t* proof);
/* Warm every lane for the given proving keys' shapes before serving: one eager commit + prove
 * of each shape sizes the lane's scratch and pinned buffers, a second captures the shape's prove
 * into a CUDA graph that later jobs of that shape replay.  Synthetic inputs; nothing is returned.
 * Call with no job queued or running (else LGS_ERR_BAD_ARG).  No reference counterpart. */
lgs_status lgs_engine_prepare(lgs_engine* e, const lgs_pk* const* pks, size_t npk);
/* Jobs waiting for a lane, and the device bytes reserved by running jobs. */
lgs_status lgs_engine_pending(lgs_engine* e, size_t* queued, size_t* running_bytes);
/* lgs_tune on every lane (same names and limits).  Small jobs run side by side when their
 * kernels leave SMs free: a lower hash_ctas / sumcheck_blocks cap trades one job's latency for
 * the batch's throughput.  Call with no job queued or running (else LGS_ERR_BAD_ARG); a
 * sumcheck_blocks change drops the lanes' captured prove graphs (lgs_engine_prepare again).
 * No reference counterpart. */
lgs_status lgs_engine_tune(lgs_engine* e, const char* name, uint64_t value);

/* ---- measurement (no counterpart in the reference, whose benches use wall-clock timers,
 * pcs/benches/ligesis.rs:27-45) ---- */

/* enable != 0: record CUDA events around each device stage of later calls on this context
 * (and clear the totals); 0: stop.  Stages: commit_upload, rs_encode, subset_sum_hash,
 * merkle_h, upload_and_rs_encode (host f), prove_device, and the host phases host_plan,
 * host_enqueue, host_wait, host_assemble.  enable = 2 also records the prove's timeline: event
 * nodes at its branch boundaries, captured into its graph, reported as "tl:<mark>" = ms from the
 * prove's start to that point (marks: prefix_end, A1_abar_commit_end, ..., join, end). */
lgs_status lgs_profile(lgs_ctx* ctx, int enable);
/* Total device milliseconds and number of timed calls of one stage since lgs_profile(ctx, 1). */
lgs_status lgs_profile_get(lgs_ctx* ctx, const char* stage, double* total_ms, uint64_t* count);
/* Names of the stages with totals since lgs_profile(ctx, 1|2), one per line ("tl:<mark>" for
 * timeline marks); *needed receives the buffer size that holds them all (with the NUL). */
lgs_status lgs_profile_names(lgs_ctx* ctx, char* buf, size_t cap, size_t* needed);
/* Launch choices of this context's kernels, picked by the autotuner (ligesis_b200/autotune.py;
 * no counterpart in the reference, which has no kernels).  0 restores the built-in default.
 *   "hash_ctas"        persistent CTAs of the subset-sum hash (default one per SM); fewer leave
 *                      SMs to the prove that runs beside the commit's hash
 *   "sumcheck_blocks"  grid cap of the multi-CTA sumcheck passes (at most 296)
 *   "hash_groups"      commits of host polynomials: digest the codeword in this many row
 *                      groups (1..8) as their RS encoding finishes, under the upload
 *   "witness_path"     lgs_linear_witness: 0 the int8 tensor cores whenever every activation
 *                      fits 24 and every weight 16 signed bits (else the CUDA cores), 1 always
 *                      the CUDA cores
 *   "upload_block_bytes" commits of host polynomials: the least bytes per row block of the
 *                      upload pipelined with the RS encoding (0: 1 MB; an engine's lanes
 *                      start at 4 MB)
 *   "upload_tail_rows" commits of host polynomials: rows of the last of those row blocks, whose
 *                      RS encoding the prove waits for after the upload (0, or a whole equal
 *                      share or more: equal blocks)
 *   "witness_ctas"     lgs_linear_witness on the tensor cores: the resident CTAs its work plan
 *                      assumes (whole waves of output tiles, the remaining tiles split over K
 *                      to fill the last wave); 0 the GPU's own count
 * Results do not depend on them.  Unknown names: LGS_ERR_BAD_ARG. */
lgs_status lgs_tune(lgs_ctx* ctx, const char* name, uint64_t value);
lgs_status lgs_tune_get(lgs_ctx* ctx, const char* name, uint64_t* value);
/* Clock-cycle budget of the bounded device waits in the kernels this context launches (the
 * subset-sum hash's pipeline waits; no counterpart in the reference, whose code has no device
 * waits).  0 restores the default of about 2 s.  A budget shorter than the awaited event makes
 * the wait give up: the kernel stops its roles, waits for the tensor-core work and the copies it
 * has in flight (those two drains keep the default budget), frees its tensor memory and returns,
 * and the call reports LGS_ERR_DEVICE_TIMEOUT; the context stays usable.  For tests of that
 * path. */
lgs_status lgs_set_wait_budget(lgs_ctx* ctx, uint64_t cycles);
/* Number of kernels this library has launched in this process. */
uint64_t lgs_launch_count(void);
/* The int8 tensor-core rate the subset-sum hash is measured against: every SM issues `iters` x 4
 * back-to-back tcgen05.mma.kind::i8 M128 N256 K32 from shared memory (the hash's MMA shape);
 * *tops receives the best of three timed launches in TOP/s (2 ops per multiply-add). */
lgs_status lgs_tensor_peak_i8(lgs_ctx* ctx, unsigned iters, double* tops);
/* The arithmetic floor of the commitment's RS encoding: device-wide rates, per second, of the
 * radix-8 DFT every stage of the encoding runs and of its twiddle multiplications, each from a
 * kernel that keeps eight values per thread in registers for `iters` iterations (no memory
 * traffic; best of three timed launches).  No reference counterpart. */
lgs_status lgs_rs_alu_rates(lgs_ctx* ctx, unsigned iters, double* radix8_per_s,
                            double* mul_per_s);

/* ---- the individual device operations of the path (host buffers in and out) ---- */

/* Radix2Dit::dft of `batch` vectors (p3-dft 0.5.3; pcs/src/ligesis.rs:231-235): in holds
 * batch x n_in BF, each zero-padded to 2^log_size; out holds batch x 2^log_size. */
lgs_status lgs_dft(lgs_ctx* ctx, const uint64_t* in, size_t n_in, size_t batch,
                   unsigned log_size, uint64_t* out);
/* SubsetSumHash::hash_columns (pcs/src/subset_sum.rs:58-67) on bit columns given as the RS
 * codeword: cw is m x cols BF; column j's bits are bit b of cw[i][j] at row 64 i + b.
 * A is 32 x 64m; H receives 32 x cols. */
lgs_status lgs_subset_sum_hash(lgs_ctx* ctx, const uint64_t* A, size_t m, const uint64_t* cw,
                               size_t cols, uint64_t* H);
/* MerkleTreeProver::new + commit (utils/src/merkle.rs:49-85): leaves are nleaves x words
 * u64 serialized little-endian; nleaves a power of two, words * 8 <= 1024. */
lgs_status lgs_merkle_root(lgs_ctx* ctx, const uint64_t* leaves, size_t nleaves, unsigned words,
                           uint8_t root[32]);
/* sumcheck::prove (utils/src/sumcheck.rs:37-84): d factors (1..3) of 2^k EF each,
 * factor-major; challenges: k EF (the oracle fields it draws, in order).  rounds_out receives
 * k x (d+1) EF, finals_out d EF. */
lgs_status lgs_sumcheck_prove(lgs_ctx* ctx, const uint64_t* polys, unsigned d, unsigned k,
                              const uint64_t* challenges, uint64_t* rounds_out,
                              uint64_t* finals_out);
/* MlPoly::eval (utils/src/poly.rs:7-18): 2^k EF at a k-EF point. */
lgs_status lgs_mle_eval(lgs_ctx* ctx, const uint64_t* evals, unsigned k, const uint64_t* point,
                        uint64_t out[2]);
/* MlPoly::new_eq (utils/src/poly.rs:44-53): 2^k EF. */
lgs_status lgs_new_eq(lgs_ctx* ctx, const uint64_t* point, unsigned k, uint64_t* out);

/* ---- device-resident forms of the same operations (inputs already in HBM of the context's
 * device, all canonical; the work is enqueued on the context's stream, lgs_ctx_stream, and the
 * call returns without waiting for it) ---- */
/* sumcheck::prove (utils/src/sumcheck.rs:37-84) on d factors of 2^k EF stored factor-major at
 * polys_dev.  Like the reference's prove, which takes its polys by value, it consumes them:
 * the factors are folded in place.  rounds_out_dev: k x (d+1) EF; finals_out_dev: d EF. */
lgs_status lgs_sumcheck_prove_dev(lgs_ctx* ctx, uint64_t* polys_dev, unsigned d, unsigned k,
                                  const uint64_t* challenges_dev, uint64_t* rounds_out_dev,
                                  uint64_t* finals_out_dev);
/* MlPoly::new_eq (utils/src/poly.rs:44-53): 2^k EF written to out_dev. */
lgs_status lgs_new_eq_dev(lgs_ctx* ctx, const uint64_t* point_dev, unsigned k, uint64_t* out_dev);
/* MlPoly::fold (utils/src/poly.rs:33-42) of the np lowest variables (1 <= np <= 8) at
 * point_dev[0 .. np): 2^k EF in, 2^(k-np) EF out. */
lgs_status lgs_mle_fold_dev(lgs_ctx* ctx, const uint64_t* evals_dev, unsigned k,
                            const uint64_t* point_dev, unsigned np, uint64_t* out_dev);
/* MlPoly::eval (utils/src/poly.rs:7-18): one EF written to out_dev. */
lgs_status lgs_mle_eval_dev(lgs_ctx* ctx, const uint64_t* evals_dev, unsigned k,
                            const uint64_t* point_dev, uint64_t* out_dev);

/* ---- allocation-free variant (no counterpart in the reference) ----
 * The product sumcheck prover (the same computation as lgs_sumcheck_prove) for callers that
 * must not allocate device memory: processes whose HBM is owned by another allocator, and
 * serving loops that cannot afford cudaMalloc's device-wide synchronisation.  All pointers are
 * device pointers on the current device; polys holds d factors of 2^k EF, factor-major, and
 * challenges_dev k EF, all canonical (< p: unlike lgs_sumcheck_prove, this call does not reduce
 * its inputs); polys is only read; the work is enqueued on `stream` (a cudaStream_t, NULL for
 * the legacy default stream) and the call returns without waiting for it.  Limits: 1 <= d <= 3,
 * 1 <= k <= 16, else LGS_ERR_BAD_SHAPE.  The working storage is a fixed 3.3 MiB device array
 * that every GPU loading the library holds until exit; the first call in a CUDA context (a
 * device's primary context, normally) looks up the array's address there and caches it for that
 * context (make that call before any stream capture); calls that overlap on the GPU race on it.
 * It allocates nothing: no cudaMalloc, cudaFree or allocating library call. */
lgs_status lgs_sumcheck_prove_noalloc(const uint64_t* polys_dev, unsigned d, unsigned k,
                                      const uint64_t* challenges_dev, uint64_t* rounds_out_dev,
                                      uint64_t* finals_out_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LGS_H */
