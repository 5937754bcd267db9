// Host-side state of the prover library: device buffers, the per-context arena, the proving
// key and commitment data (the reference's ProvingKey / CommitData, pcs/src/ligesis.rs:67-97)
// kept resident on the device.
#pragma once
#include <chrono>
#include <memory>
#include <string>
#include <vector>

#include "../../include/lgs.h"
#include "kernels.cuh"
#include "proof.hpp"

namespace lgs {

// Device buffer from the device's stream-ordered memory pool (cudaMallocAsync on the owning
// context's stream).  The pool keeps freed memory cached (the context raises its release
// threshold), so a commitment allocated and freed per proof costs no cudaMalloc / device sync.
// Page-locked host buffer that only grows (cudaMallocHost / cudaFreeHost).
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  void reserve(size_t b) {
    if (b <= bytes) return;
    release();
    size_t want = 4096;
    while (want < b) want <<= 1;
    LGS_CUDA(cudaMallocHost(&p, want));
    bytes = want;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
  }
  ~PinnedBuf() { release(); }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

// A non-blocking stream per device that lives as long as the process: the stream on which
// buffers that outlive their context are freed.
cudaStream_t release_stream(int device);

struct DevMem {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  DevMem() = default;
  DevMem(size_t b, cudaStream_t s) { alloc(b, s); }
  void alloc(size_t b, cudaStream_t s) {
    release();
    st = s;
    if (b) LGS_CUDA(cudaMallocAsync(&p, b, st));
    bytes = b;
  }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
  }
  // For buffers that may outlive the context that allocated them (proving keys, commitment
  // data): free them on `s` (release_stream) instead of the context's stream.  Every API call
  // synchronises its streams before returning, so no work of the owning context still uses the
  // buffer when it is freed.
  void detach(cudaStream_t s) { st = s; }
  ~DevMem() { release(); }
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  DevMem(DevMem&& o) noexcept : p(o.p), bytes(o.bytes), st(o.st) { o.p = nullptr, o.bytes = 0; }
  DevMem& operator=(DevMem&& o) noexcept {
    release();
    p = o.p, bytes = o.bytes, st = o.st;
    o.p = nullptr, o.bytes = 0;
    return *this;
  }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

// Device buffers and events of commitment data, recycled per device: a commitment is created and
// freed once per proof, and returning its buffers to the stream-ordered pool (and allocating them
// again) put driver calls that can stall for milliseconds on that path.  A buffer is handed back
// only when no work uses it any more, so a later commitment may take it on any stream.  At most
// CACHE_BYTES stay cached per device; beyond that buffers go back to the pool.
struct RecycledBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int device = -1;
  RecycledBuf() = default;
  RecycledBuf(const RecycledBuf&) = delete;
  RecycledBuf& operator=(const RecycledBuf&) = delete;
  // A buffer of exactly `b` bytes on `device` (reused if one is cached), stream-ordered on `s`
  // when newly allocated.
  void acquire(size_t b, int dev, cudaStream_t s);
  void release();
  ~RecycledBuf() { release(); }
  template <class T>
  T* as() const {
    return (T*)p;
  }
};
cudaEvent_t recycled_event();
void recycle_event(cudaEvent_t e);

// Bump allocator for per-call device scratch.  A call that outgrows the buffer takes extra
// pool allocations; the next call starts from one buffer of the largest size seen, so
// steady-state calls allocate nothing.
struct Arena {
  DevMem mem;
  std::vector<DevMem> overflow;
  size_t off = 0, hwm = 0;
  cudaStream_t st = nullptr;
  bool frozen = false;  // set while a graph is captured: growing would need a synchronisation
  void begin() {
    if (!overflow.empty() || hwm > mem.bytes) {
      overflow.clear();
      mem.alloc(hwm + (hwm >> 4), st);
    }
    off = 0;
  }
  template <class T>
  T* get(size_t count) {
    size_t b = (count * sizeof(T) + 255) & ~(size_t)255;
    if (b == 0) b = 256;
    T* r;
    if (off + b <= mem.bytes) {
      r = (T*)((char*)mem.p + off);
    } else {
      if (frozen) throw std::logic_error("arena: growth while capturing a graph");
      // Grown mid-call: make the new block usable from every stream of the context at once.
      overflow.emplace_back(b, st);
      LGS_CUDA(cudaStreamSynchronize(st));
      r = overflow.back().as<T>();
    }
    off += b;
    hwm = std::max(hwm, off);
    return r;
  }
};

struct BasefoldDev {
  u64* codes = nullptr;  // leaf-major: L x 2^li elements (1 u64 per BF, 2 per EF)
  u32* nodes = nullptr;  // Merkle tree, layer-major, 8 words per node
  const u64* poly = nullptr;
  int is_ef = 0;
  unsigned li = 0, num_vars = 0;
  size_t L = 0;
  unsigned leaf_words() const { return (1u << li) * (is_ef ? 2 : 1); }
  size_t node_count() const { return 2 * L - 1; }
};

// Optional per-stage device timing: CUDA events recorded on the context stream around each
// stage, read back after the call's final synchronisation.
struct Profiler {
  struct Rec {
    std::string name;
    cudaEvent_t a, b;
  };
  bool on = false;
  std::vector<Rec> pending;
  std::vector<std::pair<std::string, std::pair<double, uint64_t>>> totals;
  void add(const std::string& name, double ms) {
    for (auto& t : totals)
      if (t.first == name) {
        t.second.first += ms;
        t.second.second += 1;
        return;
      }
    totals.push_back({name, {ms, 1}});
  }
  void flush() {  // call only after the stream has been synchronised
    for (auto& r : pending) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) add(r.name, ms);
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    pending.clear();
  }
};

struct StageTimer {
  Profiler* p;
  cudaStream_t st;
  Profiler::Rec rec;
  StageTimer(Profiler& prof, cudaStream_t s, const char* name) : p(prof.on ? &prof : nullptr), st(s) {
    if (!p) return;
    rec.name = name;
    LGS_CUDA(cudaEventCreate(&rec.a));
    LGS_CUDA(cudaEventCreate(&rec.b));
    LGS_CUDA(cudaEventRecord(rec.a, st));
  }
  void stop() {
    if (!p) return;
    if (cudaEventRecord(rec.b, st) == cudaSuccess) p->pending.push_back(rec);
    p = nullptr;
  }
  ~StageTimer() { stop(); }
};

// A prove captured as a CUDA graph for one shape.  Valid while the context's arena block and
// pinned transfer buffers are the ones it was captured with.
struct ProveGraph {
  unsigned log_m = 0, log_n = 0;
  size_t need = 0;  // arena bytes one prove of this shape uses (measured by an eager prove)
  const void* arena = nullptr;
  size_t arena_bytes = 0;
  const void* up = nullptr;
  const void* down = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t launches = 0;  // kernels per replay
  bool timeline = false;  // captured with the timeline event nodes of profile level 2
};

// Host-side phases of one call (planning, enqueueing, waiting, assembling), recorded in the
// same profile as the device stages while profiling is on.
struct HostClock {
  Profiler* p;
  std::chrono::steady_clock::time_point t;
  explicit HostClock(Profiler& prof)
      : p(prof.on ? &prof : nullptr), t(std::chrono::steady_clock::now()) {}
  void lap(const char* name) {
    if (!p) return;
    const auto now = std::chrono::steady_clock::now();
    p->add(name, std::chrono::duration<double, std::milli>(now - t).count());
    t = now;
  }
};

}  // namespace lgs

struct lgs_ctx {
  static constexpr int NSIDE = 12;  // side streams for the independent branches of prove
  static constexpr int RING = 3;    // pinned chunks for staged uploads of host polynomials
  static constexpr size_t RING_CHUNK = (size_t)8 << 20;
  int device = 0;
  cudaStream_t st = nullptr;
  cudaStream_t side[NSIDE] = {};
  static constexpr int NSIDE_HI = 3;  // high-priority side streams for the critical branches
  cudaStream_t side_hi[NSIDE_HI] = {};
  cudaEvent_t ev_fork2 = nullptr;
  // The commit's hash and Merkle tree run on hs after the codeword is ready (ev_cw), so a prove
  // that follows overlaps them; only its final gather waits for the commitment's tree.
  cudaStream_t hs = nullptr;
  cudaEvent_t ev_cw = nullptr;
  cudaEvent_t ev_done[NSIDE] = {};
  cudaEvent_t ev_fork = nullptr;
  static constexpr int ROW_BLOCKS = 8;  // row blocks of a host upload pipelined with RS encoding
  cudaEvent_t ev_rows[ROW_BLOCKS] = {};
  cudaEvent_t ev_rs[ROW_BLOCKS] = {};  // RS encoding of row block b done (host-rows commit)
  lgs::DevMem tw;
  lgs::DevMem rs_tw;  // twiddles of the row RS encoding (rs_dft.cu)
  lgs::DevMem hash_scr;  // digest slices of a split subset-sum hash (used on hs only)
  lgs::Arena arena;
  lgs::Profiler prof;
  // Profile level 2: event-record nodes at the prove's branch boundaries (captured into its
  // graph), read back as "tl:<mark>" = ms since the prove's start.
  int prof_level = 0;
  static constexpr int TL_MAX = 96;
  cudaEvent_t tl_ev[TL_MAX] = {};
  std::vector<std::string> tl_names;
  unsigned tl_count = 0;  // marks recorded inside the prove's graph
  lgs::DevMem err;  // device error word of bounded-wait kernels (0 = ok)
  uint64_t wait_cycles = 0;  // budget of those waits in clock cycles (0 = default; lgs_set_wait_budget)
  // Launch choices the autotuner sets (lgs_tune): 0 = the built-in default.
  unsigned hash_ctas = 0;        // persistent CTAs of the subset-sum hash (default: one per SM)
  unsigned sumcheck_blocks = 0;  // grid cap of the multi-CTA sumcheck passes (<= SC_MAX_BLOCKS)
  unsigned hash_groups = 0;      // host-rows commit: hash launches over row groups (0: default)
  unsigned witness_path = 0;     // linear witness: 0 tensor cores when the operands fit, 1 CUDA cores
  unsigned witness_ctas = 0;     // linear witness: resident CTAs its work plan assumes (0: the GPU's)
  size_t upload_block = 0;       // host-rows commit: least bytes per row block (0: 1 MB)
  size_t upload_tail = 0;        // host-rows commit: rows of the last row block (0: equal)
  // Pinned host memory: every transfer of a call is asynchronous, so the host enqueues a whole
  // commit or prove without waiting for the device and synchronises once at the end.
  lgs::PinnedBuf up;    // the parameter blob of one prove (one host-to-device copy)
  lgs::PinnedBuf down;  // the staging area one prove reads back
  lgs::PinnedBuf tail;  // error word and root of the last commit
  lgs::PinnedBuf ring[RING];
  cudaEvent_t ring_ev[RING] = {};
  unsigned ring_next = 0;
  bool copy_pool = true;  // staged uploads use the process's copy threads (engine lanes: no)
  bool use_graphs = true;
  std::vector<lgs::ProveGraph> graphs;
  std::vector<uint8_t> proof_buf;   // the last proof returned by lgs_prove
};

struct lgs_pk {
  lgs::Shape shape;
  bool commit_only = false;  // lgs_setup_commit_only: no Basefold commitment of A, no prove
  lgs::DevMem A;      // 32 x W canonical u64, row-major (the flat A-bar of subset_sum.rs:73-79)
  lgs::DevMem alimb;  // 256 x W bytes: byte l of A[r][k] at row 8r + l
  alignas(64) unsigned char tmap[128];  // TMA descriptor of alimb (CUtensorMap)
  lgs::DevMem a_codes, a_nodes;
  lgs::BasefoldDev a_state;
  lgs::Hash32 com_a;
};

struct lgs_commit_data {
  const uint64_t* fdev() const { return f_lent ? f_lent : f.as<uint64_t>(); }
  lgs::Shape shape;
  cudaEvent_t done = nullptr;  // recorded after the commit's last copy (asynchronous commits)
  bool root_ready = false;
  lgs::RecycledBuf f;      // m x n (unused when the caller lends its device copy)
  const uint64_t* f_lent = nullptr;  // the caller's device f, kept alive and unchanged by it
  lgs::RecycledBuf cw;     // m x 2n RS codeword F' (its bits are B)
  lgs::RecycledBuf H;      // 32 x 2n digest
  lgs::RecycledBuf nodes;  // column Merkle tree over H
  lgs::Hash32 root;
  ~lgs_commit_data() {
    if (done) lgs::recycle_event(done);
  }
};

// A standalone Basefold commitment (pcs/src/basefold.rs:46-58 BasefoldProverState) resident on
// the device: the polynomial, its interleaved codewords (leaf-major) and their Merkle tree.
struct lgs_basefold {
  int device = 0;
  lgs::DevMem poly;   // 2^n values: BF (1 u64) or EF (2 u64), canonical
  lgs::DevMem codes;  // L x 2^li values, leaf-major
  lgs::DevMem nodes;  // Merkle tree over the L leaves
  lgs::BasefoldDev st;
  unsigned code_rate = 0;
  lgs::Hash32 root;
};

namespace lgs {
// The prover's stages (prover.cu).  commit_dev with finish = false only enqueues: commit_finish
// (or any later synchronisation of the context followed by commit_finish) completes it.
void ctx_init(lgs_ctx* c, int device);
// commit_only: any shape the commit kernels take (log_n >= 7, log_m <= 13); the key then holds
// only A and its limbs, and cannot be used by prove.
void setup_dev(lgs_ctx* c, unsigned log_m, unsigned log_n, const u64* A_host, lgs_pk* pk,
               bool commit_only = false);
void commit_dev(lgs_ctx* c, const lgs_pk* pk, const u64* f, bool f_on_device, lgs_commit_data* cd,
                bool finish = true);
void commit_finish(lgs_ctx* c, lgs_commit_data* cd);
void commit_root(lgs_ctx* c, lgs_commit_data* cd);
// Standalone Basefold (pcs/src/basefold.rs:309-516): commit_{base,ext}_on_domain of a host
// polynomial and Basefold::prove at a point, the proof encoded as in proof.hpp ("LGSB").
void basefold_commit_dev(lgs_ctx* c, const u64* poly, size_t len, int is_ef, unsigned code_rate,
                         unsigned li, lgs_basefold* out);
void basefold_prove_dev(lgs_ctx* c, const lgs_basefold* b, const u64* point, size_t plen,
                        const u64* fields, size_t nfields, const uint64_t* ints, size_t nints,
                        uint64_t cursors[2], std::vector<uint8_t>* proof_out);
int basefold_verify_host(const Hash32& root, const u64* point, size_t plen, const uint8_t* proof,
                         size_t proof_len, const u64* fields, size_t nfields, const uint64_t* ints,
                         size_t nints, uint64_t cursors[2]);
void prove_dev(lgs_ctx* c, const lgs_pk* pk, const lgs_commit_data* cd, const u64* z_host,
               size_t zlen, const u64* fields_host, size_t nfields, const uint64_t* ints_host,
               size_t nints, uint64_t cursors[2], std::vector<uint8_t>* proof_out);
// Host-to-device copy of a (pageable) host buffer through the context's pinned ring.
void h2d_staged(lgs_ctx* c, void* dst, const void* src, size_t bytes, cudaStream_t st);
// GKR fraction sum (logup/src/frac_sum.rs:110-161) and GKR-LogUp lookup
// (logup/src/lookup.rs:119-143) on the device (frac_sum.cu), proofs encoded "LGSF" / "LGSL"; and
// their host verifiers (logup_verify.cpp).  Inputs are EF arrays (2 u64 per value) on the host,
// or on the device when on_device; `cursor` is the oracle's fields cursor.
void frac_sum_prove_dev(lgs_ctx* c, const u64* p, const u64* q, size_t n, bool on_device,
                        const u64* fields, size_t nfields, uint64_t* cursor,
                        std::vector<uint8_t>* proof_out, u64* point_out, u64* claim_out);
void lookup_prove_dev(lgs_ctx* c, const u64* a, size_t m, const u64* t, const u64* e, size_t n,
                      bool on_device, const u64* fields, size_t nfields, uint64_t* cursor,
                      std::vector<uint8_t>* proof_out, u64* zq_out, u64* zt_out);
int frac_sum_verify_host(const uint8_t* proof, size_t len, const u64* fields, size_t nfields,
                         uint64_t* cursor, u64* point, size_t point_cap, u64* claim);
int lookup_verify_host(const uint8_t* proof, size_t len, const u64* fields, size_t nfields,
                       uint64_t* cursor, u64* zq, size_t zq_cap, u64* zt, size_t zt_cap,
                       u64* vals);
// proofsys' rescaled linear-layer witness (witness.cu): Q, REM = floor_div(X W, divisor),
// Y = Q + bias, Y_field = encode_i64(Y); row-major i64 arrays, on the host or (on_device) the device.
// The layer's contraction on the int8 tensor cores (witness_tc.cu), on device operands; sets
// *drange when an operand is outside its limb encoding (nothing usable is written then).
void linear_witness_tc(lgs_ctx* c, const int64_t* dx, size_t rows, size_t inner,
                       const int64_t* dw, size_t cols, bool w_transposed, const int64_t* db,
                       int64_t divisor, int64_t* dq, int64_t* dr, int64_t* dy, uint64_t* df,
                       int* derr, int* drange);
void linear_witness_dev(lgs_ctx* c, const int64_t* x, size_t rows, size_t inner, const int64_t* w,
                        size_t cols, bool w_transposed, const int64_t* bias, int64_t divisor,
                        bool on_device, int64_t* q, int64_t* rem, int64_t* y, uint64_t* y_field);
// proofsys' layer-norm witness (witness.cu): per row sum_x, sum_x2, var_sum, std; per entry
// dividend, quotient, output.
void layer_norm_witness_dev(lgs_ctx* c, const int64_t* x, size_t rows, size_t d,
                            const int64_t* gain, const int64_t* bias, bool on_device,
                            int64_t* const per_row[4], int64_t* const per_entry[3]);
// proofsys' causal softmax witness and lookup gather (witness.cu).
void softmax_witness_dev(lgs_ctx* c, const int64_t* scores, unsigned heads, unsigned n,
                         const int64_t* lut, size_t lut_len, int64_t offset, int64_t scale,
                         bool on_device, int64_t* x_max, int64_t* ex, int64_t* sum_exp,
                         int64_t* prob);
void lut_gather_dev(lgs_ctx* c, const int64_t* v, size_t count, const int64_t* lut,
                    size_t lut_len, int64_t offset, bool on_device, int64_t* out);
lgs_status set_error(lgs_status s, const std::string& msg);
lgs_status status_of_current_exception();
}  // namespace lgs
