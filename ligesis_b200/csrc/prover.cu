// The LigeSIS prover on one GPU: Ligesis::setup / commit / prove (pcs/src/ligesis.rs:239-549)
// with the Basefold interleaved commit (pcs/src/basefold.rs:257-382) and shared-domain batched
// open (pcs/src/basefold.rs:648-856).  Every challenge of the pre-drawn oracle is known before
// the first kernel runs, so `prove` uploads one parameter block, enqueues the whole dataflow on
// the context stream, and reads back one staging buffer from which the proof is assembled.
#include <functional>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>

#include "prover.cuh"

namespace lgs {

namespace {

void h2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes) LGS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
}
void d2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes) LGS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st));
}

// Basefold commit of `poly` (len elements, BF or EF) split into 2^li interleaved chunks
// (MlPoly::split, utils/src/poly.rs:20-31), each zero-padded to len/2^li << code_rate and
// DFT'd; leaves are the columns across chunks.  `out` receives codes (leaf-major) and the tree.
void bf_commit(lgs_ctx* c, const u64* poly, int is_ef, size_t len, unsigned li,
               unsigned code_rate, BasefoldDev* out, cudaStream_t st) {
  Arena& ar = c->arena;
  const size_t rows = len >> li;
  const size_t cols = ((size_t)1 << li) * (is_ef ? 2 : 1);
  const size_t L = rows << code_rate;
  const unsigned logL = ilog2(L);
  u64* tT = ar.get<u64>(cols * rows);
  u64* cT = ar.get<u64>(cols * L);
  u64* scr = logL > 12 ? ar.get<u64>(cols * L) : nullptr;
  transpose_u64(poly, tT, rows, cols, 1, st);
  // large transforms use the row kernels (one CTA per four columns of a row, which fills the
  // GPU only with many rows); the prove's small Basefold commits keep the Stockham kernels
  if (rs_dft_supported(logL, rows) && cols * L >= ((size_t)1 << 22) && cols <= 65535)
    rs_dft_rows(tT, rows, rows, cT, L, logL, cols, scr, c->rs_tw.as<u64>(), st);
  else
    ntt_batch(tT, rows, rows, cT, L, logL, cols, scr, c->tw.as<u64>(), st);
  transpose_u64(cT, out->codes, cols, L, 1, st);
  tl_mark("bf_dft_end", st);
  merkle_leaves_contig(out->codes, (unsigned)cols, L, out->nodes, st);
  tl_mark("bf_leaves_end", st);
  merkle_build_from_leaves(out->nodes, L, st);
  out->poly = poly;
  out->is_ef = is_ef;
  out->li = li;
  out->num_vars = ilog2(len);
  out->L = L;
}

// Host threads shared by every context of the process for large pageable-to-pinned copies: one
// thread's memcpy reaches a fraction of the host's memory bandwidth.
class CopyPool {
 public:
  static CopyPool& get() {
    static CopyPool* pool = new CopyPool;  // never destroyed: its threads wait until exit
    return *pool;
  }
  // memcpy split into parts of at least 1 MiB, run by the pool's threads and the caller.
  void copy(void* dst, const void* src, size_t bytes) {
    const size_t parts = std::min<size_t>(threads_.size() + 1, std::max<size_t>(1, bytes >> 20));
    if (parts <= 1) {
      std::memcpy(dst, src, bytes);
      return;
    }
    const size_t step = (bytes / parts + 63) & ~(size_t)63;
    Batch batch;
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (size_t i = 1; i < parts; ++i) {
        const size_t off = std::min(bytes, i * step);
        const size_t len = std::min(bytes, off + step) - off;
        if (len) {
          ++batch.left;
          tasks_.push_back({(char*)dst + off, (const char*)src + off, len, &batch});
        }
      }
    }
    cv_.notify_all();
    std::memcpy(dst, src, std::min(bytes, step));
    std::unique_lock<std::mutex> lk(mu_);
    batch.cv.wait(lk, [&] { return batch.left == 0; });
  }

 private:
  struct Batch {
    size_t left = 0;
    std::condition_variable cv;
  };
  struct Task {
    char* dst;
    const char* src;
    size_t len;
    Batch* batch;
  };
  CopyPool() {
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    for (unsigned i = 0; i < std::min(8u, hw / 2); ++i) {
      threads_.emplace_back([this] { run(); });
      threads_.back().detach();  // lives as long as the process
    }
  }
  void run() {
    std::unique_lock<std::mutex> lk(mu_);
    while (true) {
      cv_.wait(lk, [&] { return !tasks_.empty(); });
      Task t = tasks_.front();
      tasks_.pop_front();
      lk.unlock();
      std::memcpy(t.dst, t.src, t.len);
      lk.lock();
      if (--t.batch->left == 0) t.batch->cv.notify_all();
    }
  }
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Task> tasks_;
  std::vector<std::thread> threads_;
};

bool host_is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

}  // namespace

// Host-to-device copy of a large host array.  Page-locked memory goes straight to the DMA engine;
// pageable memory goes through the context's ring of pinned chunks (the copy pool fills chunk i
// while the DMA engine moves chunk i-1).  The caller's array is no longer read when this returns.
void h2d_staged(lgs_ctx* c, void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (host_is_pinned(src)) {
    h2d(dst, src, bytes, st);
    return;
  }
  for (size_t off = 0; off < bytes; off += lgs_ctx::RING_CHUNK) {
    const unsigned slot = c->ring_next++ % lgs_ctx::RING;
    const size_t len = std::min(lgs_ctx::RING_CHUNK, bytes - off);
    LGS_CUDA(cudaEventSynchronize(c->ring_ev[slot]));  // the slot's previous copy has landed
    c->ring[slot].reserve(lgs_ctx::RING_CHUNK);
    if (c->copy_pool)
      CopyPool::get().copy(c->ring[slot].p, (const char*)src + off, len);
    else
      std::memcpy(c->ring[slot].p, (const char*)src + off, len);
    LGS_CUDA(cudaMemcpyAsync((char*)dst + off, c->ring[slot].p, len, cudaMemcpyHostToDevice, st));
    LGS_CUDA(cudaEventRecord(c->ring_ev[slot], st));
  }
}

namespace {

Hash32 read_root(const u32* nodes, size_t nleaves, cudaStream_t st) {
  Hash32 h;
  LGS_CUDA(cudaMemcpyAsync(h.b, nodes + (2 * nleaves - 2) * 8, 32, cudaMemcpyDeviceToHost, st));
  LGS_CUDA(cudaStreamSynchronize(st));
  return h;
}

}  // namespace

cudaStream_t release_stream(int device) {
  static std::mutex mu;
  static std::vector<cudaStream_t> streams;
  std::lock_guard<std::mutex> lk(mu);
  if (device < 0) throw std::runtime_error("release_stream: bad device");
  if ((size_t)device >= streams.size()) streams.resize(device + 1, nullptr);
  if (!streams[device]) {
    int prev = 0;
    LGS_CUDA(cudaGetDevice(&prev));
    LGS_CUDA(cudaSetDevice(device));
    LGS_CUDA(cudaStreamCreateWithFlags(&streams[device], cudaStreamNonBlocking));
    LGS_CUDA(cudaSetDevice(prev));
  }
  return streams[device];
}

namespace {
constexpr size_t CACHE_BYTES = (size_t)8 << 30;
struct Cached {
  int device;
  size_t bytes;
  void* p;
};
std::mutex g_cache_mu;
std::vector<Cached> g_cache;
std::vector<cudaEvent_t> g_events;
size_t g_cached_bytes = 0;
}  // namespace

void RecycledBuf::acquire(size_t b, int dev, cudaStream_t s) {
  if (p && bytes == b && device == dev) return;
  release();
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (size_t i = 0; i < g_cache.size(); ++i)
      if (g_cache[i].device == dev && g_cache[i].bytes == b) {
        p = g_cache[i].p;
        g_cache.erase(g_cache.begin() + i);
        g_cached_bytes -= b;
        bytes = b;
        device = dev;
        return;
      }
  }
  if (b) LGS_CUDA(cudaMallocAsync(&p, b, s));
  bytes = b;
  device = dev;
}

void RecycledBuf::release() {
  if (!p) return;
  bool keep = false;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (g_cached_bytes + bytes <= CACHE_BYTES) {
      g_cache.push_back({device, bytes, p});
      g_cached_bytes += bytes;
      keep = true;
    }
  }
  if (!keep) cudaFreeAsync(p, release_stream(device));
  p = nullptr;
  bytes = 0;
}

cudaEvent_t recycled_event() {
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (!g_events.empty()) {
      cudaEvent_t e = g_events.back();
      g_events.pop_back();
      return e;
    }
  }
  cudaEvent_t e = nullptr;
  LGS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return e;
}

void recycle_event(cudaEvent_t e) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  if (g_events.size() < 256)
    g_events.push_back(e);
  else
    cudaEventDestroy(e);
}

void ctx_init(lgs_ctx* c, int device) {
  c->device = device;
  LGS_CUDA(cudaSetDevice(device));
  int prio_lo = 0, prio_hi = 0;
  LGS_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
  // the main stream and the prove's critical branches outrank the other branches
  LGS_CUDA(cudaStreamCreateWithPriority(&c->st, cudaStreamNonBlocking, prio_hi));
  for (int i = 0; i < lgs_ctx::NSIDE_HI; ++i)
    LGS_CUDA(cudaStreamCreateWithPriority(&c->side_hi[i], cudaStreamNonBlocking, prio_hi));
  LGS_CUDA(cudaEventCreateWithFlags(&c->ev_fork2, cudaEventDisableTiming));
  LGS_CUDA(cudaStreamCreateWithPriority(&c->hs, cudaStreamNonBlocking, prio_lo));
  LGS_CUDA(cudaEventCreateWithFlags(&c->ev_cw, cudaEventDisableTiming));
  // Keep freed pool memory cached so per-proof buffers are recycled without driver calls.
  cudaMemPool_t pool;
  LGS_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t thresh = UINT64_MAX;
  LGS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thresh));
  c->arena.st = c->st;
  for (int i = 0; i < lgs_ctx::NSIDE; ++i) {
    LGS_CUDA(cudaStreamCreateWithFlags(&c->side[i], cudaStreamNonBlocking));
    LGS_CUDA(cudaEventCreateWithFlags(&c->ev_done[i], cudaEventDisableTiming));
  }
  LGS_CUDA(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  for (int i = 0; i < lgs_ctx::ROW_BLOCKS; ++i) {
    LGS_CUDA(cudaEventCreateWithFlags(&c->ev_rows[i], cudaEventDisableTiming));
    LGS_CUDA(cudaEventCreateWithFlags(&c->ev_rs[i], cudaEventDisableTiming));
  }
  for (int i = 0; i < lgs_ctx::RING; ++i)
    LGS_CUDA(cudaEventCreateWithFlags(&c->ring_ev[i], cudaEventDisableTiming));
  c->tail.reserve(64);
  c->tw.alloc(((size_t)1 << TW_LOG) * sizeof(u64), c->st);
  c->err.alloc(sizeof(int), c->st);
  LGS_CUDA(cudaMemsetAsync(c->err.p, 0, sizeof(int), c->st));
  if (tensor_map_bytes() > sizeof(((lgs_pk*)nullptr)->tmap))
    throw std::runtime_error("tensor map larger than its slot");
  build_twiddles(c->tw.as<u64>(), c->st);
  c->rs_tw.alloc(rs_tables_elems() * sizeof(u64), c->st);
  build_rs_tables(c->rs_tw.as<u64>(), c->tw.as<u64>(), c->st);
  LGS_CUDA(cudaStreamSynchronize(c->st));
}

void setup_dev(lgs_ctx* c, unsigned log_m, unsigned log_n, const u64* A_host, lgs_pk* pk,
               bool commit_only) {
  Shape s{log_m, log_n};
  if (commit_only) {
    if (log_m > 13 || log_n < 7)
      throw ShapeError("commit-only key: needs log_m <= 13 and log_n >= 7");
  } else if (!s.eval_ok()) {
    throw ShapeError("batched LigeSIS needs the {A, B_I, a} var counts within LOG_INTERLEAVE");
  }
  pk->shape = s;
  pk->commit_only = commit_only;
  const size_t W = s.W(), len = (size_t)DIGEST_ROWS * W;
  c->arena.begin();
  pk->A.alloc(len * 8, c->st);
  pk->A.detach(release_stream(c->device));
  std::vector<u64> canon(A_host, A_host + len);
  for (auto& x : canon) x = gl_canon(x);
  h2d(pk->A.p, canon.data(), len * 8, c->st);
  pk->alimb.alloc(len * 8, c->st);
  pk->alimb.detach(release_stream(c->device));
  alimb_from_a(pk->A.as<u64>(), pk->alimb.as<uint8_t>(), W, c->st);
  make_alimb_tmap(pk->alimb.as<uint8_t>(), W, pk->tmap);
  if (commit_only) {
    LGS_CUDA(cudaStreamSynchronize(c->st));
    return;
  }
  const unsigned li = s.li(s.na());
  const size_t L = (len >> li) << CODE_RATE;
  pk->a_codes.alloc(L * ((size_t)1 << li) * 8, c->st);
  pk->a_codes.detach(release_stream(c->device));
  pk->a_nodes.alloc((2 * L - 1) * 32, c->st);
  pk->a_nodes.detach(release_stream(c->device));
  pk->a_state.codes = pk->a_codes.as<u64>();
  pk->a_state.nodes = pk->a_nodes.as<u32>();
  bf_commit(c, pk->A.as<u64>(), 0, len, li, CODE_RATE, &pk->a_state, c->st);
  pk->com_a = read_root(pk->a_state.nodes, L, c->st);
}

// Ligesis::commit (pcs/src/ligesis.rs:277-325): RS-encode rows, hash B's columns, Merkle the
// digest columns.  `f` may be a host or a device pointer (f_on_device).
void commit_dev(lgs_ctx* c, const lgs_pk* pk, const u64* f, bool f_on_device,
                lgs_commit_data* cd, bool finish) {
  const Shape& s = pk->shape;
  const size_t m = s.m(), n = s.n(), two_n = 2 * n;
  if (two_n % 128) throw ShapeError("commit: 2n must be a multiple of 128");
  HostClock hc(c->prof);
  cd->shape = s;
  c->arena.begin();
  if (!cd->f_lent) cd->f.acquire(m * n * 8, c->device, c->st);
  cd->cw.acquire(m * two_n * 8, c->device, c->st);
  cd->H.acquire(DIGEST_ROWS * two_n * 8, c->device, c->st);
  cd->nodes.acquire((2 * two_n - 1) * 32, c->device, c->st);
  const unsigned logN = ilog2(two_n);
  u64* scr = logN > 12 ? c->arena.get<u64>(m * two_n) : nullptr;
  const bool rows_path = rs_dft_supported(logN, n);
  hc.lap("host_commit_alloc");
  bool hashed = false;  // the digest was built row group by row group under the upload
  if (!f_on_device && !cd->f_lent && rows_path && m >= 2) {
    // Host rows: the upload of row block b + 1 overlaps the RS encoding of block b.  Page-locked
    // f is copied by the DMA engine on a side stream; pageable f goes through the pinned ring on
    // the context stream, where the host-side staging of the next block is the slower part.
    StageTimer t(c->prof, c->st, "upload_and_rs_encode");
    // enough row blocks that the upload of each overlaps the encoding of the one before, but
    // none smaller than upload_block (1 MB by default: a block costs a few calls and two
    // launches, which a smaller block's overlap does not pay back; engine lanes use 4 MB, their
    // jobs overlapping each other instead)
    const size_t min_block = c->upload_block ? c->upload_block : ((size_t)1 << 20);
    unsigned nb = (unsigned)std::min<size_t>(lgs_ctx::ROW_BLOCKS, m);
    while (nb > 1 && m * n * 8 / nb < min_block) nb >>= 1;
    const size_t share = m / nb;  // m and nb are powers of two
    // Row block b holds rows [brow[b], brow[b + 1]): equal blocks, or with upload_tail_rows
    // below an equal share a last block of that many rows (even, at least 2) and the rest in
    // even sizes.  The prove waits for the last block's RS encoding after its upload lands, but
    // a short block does not shorten that wait in proportion (the encoding's grid is over rows),
    // and on B200 at 2^7 x 2^17 a 4-row tail made the host-input step slower (3.58 vs 3.51 ms).
    size_t brow[lgs_ctx::ROW_BLOCKS + 1];
    brow[0] = 0;
    if (nb > 1 && share >= 4 && c->upload_tail && c->upload_tail < share) {
      const size_t tail = std::max<size_t>(2, c->upload_tail & ~(size_t)1);
      const size_t pairs = (m - tail) / 2, each = pairs / (nb - 1), extra = pairs % (nb - 1);
      for (unsigned b = 0; b + 1 < nb; ++b) brow[b + 1] = brow[b] + 2 * (each + (b < extra));
    } else {
      for (unsigned b = 0; b + 1 < nb; ++b) brow[b + 1] = (size_t)(b + 1) * share;
    }
    brow[nb] = m;
    const bool pinned = host_is_pinned(f);
    cudaStream_t cp = c->side[0];
    if (pinned) {
      LGS_CUDA(cudaEventRecord(c->ev_fork, c->st));  // cd->f exists on the context stream
      LGS_CUDA(cudaStreamWaitEvent(cp, c->ev_fork, 0));
    }
    // H is linear in the rows: with hash_groups = G > 1 the hash stream digests each group of
    // row blocks as soon as their RS encoding is done (write, then add; the last group also
    // hashes the leaves), so most of the hash runs under the rest of the upload.  Group g ends
    // with block (g + 1) nb / G - 1, which leaves no group empty for any G <= nb.
    unsigned groups = c->hash_groups ? std::min(c->hash_groups, nb) : 1;
    for (unsigned g = 1; g < groups; ++g)  // a group must hold whole pairs of rows
      if (brow[(size_t)g * nb / groups] % 2) {
        groups = 1;
        break;
      }
    unsigned g = 0;  // the next group to hash
    for (unsigned b = 0; b < nb; ++b) {
      const size_t rows = brow[b + 1] - brow[b], off = brow[b] * n;
      if (pinned) {
        h2d(cd->f.as<u64>() + off, f + off, rows * n * 8, cp);
        LGS_CUDA(cudaEventRecord(c->ev_rows[b], cp));
        LGS_CUDA(cudaStreamWaitEvent(c->st, c->ev_rows[b], 0));
      } else {
        h2d_staged(c, cd->f.as<u64>() + off, f + off, rows * n * 8, c->st);
      }
      rs_dft_rows(cd->f.as<u64>() + off, n, n, cd->cw.as<u64>() + brow[b] * two_n, two_n, logN,
                  (unsigned)rows, scr + brow[b] * two_n, c->rs_tw.as<u64>(), c->st);
      if (groups > 1 && b + 1 == (size_t)(g + 1) * nb / groups) {
        const size_t r0 = brow[(size_t)g * nb / groups];
        LGS_CUDA(cudaEventRecord(c->ev_rs[b], c->st));
        LGS_CUDA(cudaStreamWaitEvent(c->hs, c->ev_rs[b], 0));
        StageTimer th(c->prof, c->hs, "subset_sum_hash_rows");
        subset_sum_hash_tc(pk->tmap, cd->cw.as<u64>(), cd->H.as<u64>(), cd->nodes.as<u32>(),
                           (unsigned)m, two_n, c->err.as<int>(), c->hs, c->wait_cycles,
                           c->hash_ctas, (unsigned)r0, (unsigned)(brow[b + 1] - r0),
                           g == 0 ? 0 : (g + 1 == groups ? 3 : 1));
        hashed = true;
        ++g;
      }
    }
  } else {
    if (!cd->f_lent) {
      StageTimer t(c->prof, c->st, "commit_upload");
      if (f_on_device)
        d2d(cd->f.p, f, m * n * 8, c->st);
      else
        h2d_staged(c, cd->f.p, f, m * n * 8, c->st);
    }
    StageTimer t(c->prof, c->st, "rs_encode");
    if (rows_path)
      rs_dft_rows(cd->fdev(), n, n, cd->cw.as<u64>(), two_n, logN, m, scr, c->rs_tw.as<u64>(),
                  c->st);
    else
      ntt_batch(cd->fdev(), n, n, cd->cw.as<u64>(), two_n, logN, m, scr, c->tw.as<u64>(), c->st);
  }
  hc.lap("host_commit_rs");
  // The hash and the tree need only the codeword: they run on the hash stream, and a prove
  // enqueued next on the context stream runs beside them (its gather waits for cd->done).
  LGS_CUDA(cudaEventRecord(c->ev_cw, c->st));
  LGS_CUDA(cudaStreamWaitEvent(c->hs, c->ev_cw, 0));
  if (!hashed) {
    // digest slices of a split hash (few column tiles) live on the hash stream only
    const unsigned splits = subset_sum_hash_splits(two_n, (unsigned)m, c->hash_ctas);
    u64* slices = nullptr;
    if (splits > 1) {
      const size_t bytes = (size_t)splits * DIGEST_ROWS * two_n * 8;
      if (c->hash_scr.bytes < bytes) c->hash_scr.alloc(bytes, c->hs);
      slices = c->hash_scr.as<u64>();
    }
    StageTimer t(c->prof, c->hs, "subset_sum_hash");  // H and its Merkle leaf hashes
    subset_sum_hash_tc(pk->tmap, cd->cw.as<u64>(), cd->H.as<u64>(), cd->nodes.as<u32>(),
                       (unsigned)m, two_n, c->err.as<int>(), c->hs, c->wait_cycles, c->hash_ctas,
                       0, 0, 2, slices);
  }
  {
    StageTimer t(c->prof, c->hs, "merkle_h");
    merkle_build_from_leaves(cd->nodes.as<u32>(), two_n, c->hs);
  }
  // error word and root into pinned memory; commit_finish reads them after a synchronisation
  LGS_CUDA(cudaMemcpyAsync(c->tail.as<uint8_t>(), c->err.p, sizeof(int), cudaMemcpyDeviceToHost,
                           c->hs));
  LGS_CUDA(cudaMemcpyAsync(c->tail.as<uint8_t>() + 32, cd->nodes.as<u32>() + (2 * two_n - 2) * 8,
                           32, cudaMemcpyDeviceToHost, c->hs));
  if (!cd->done) cd->done = recycled_event();
  LGS_CUDA(cudaEventRecord(cd->done, c->hs));
  hc.lap("host_commit_hash_merkle");
  cd->root_ready = false;
  if (finish) commit_finish(c, cd);
  hc.lap("host_commit_tail");
}

// The root of an asynchronous commit: waits for its work, then reads the root node and the
// context's error word directly (the context's pinned tail may already belong to a later call).
void commit_root(lgs_ctx* c, lgs_commit_data* cd) {
  if (cd->root_ready) return;
  if (!cd->done) throw std::logic_error("commit_root: no commit was enqueued");
  LGS_CUDA(cudaEventSynchronize(cd->done));
  const size_t two_n = 2 * cd->shape.n();
  int err = 0;
  LGS_CUDA(cudaMemcpy(&err, c->err.p, sizeof(int), cudaMemcpyDeviceToHost));
  LGS_CUDA(cudaMemcpy(cd->root.b, cd->nodes.as<u32>() + (2 * two_n - 2) * 8, 32,
                      cudaMemcpyDeviceToHost));
  if (err) {
    LGS_CUDA(cudaMemset(c->err.p, 0, sizeof(int)));
    throw DeviceTimeout("subset-sum hash: a bounded device wait gave up (code " +
                        std::to_string(err) + ")");
  }
  cd->root_ready = true;
}

// Completes commit_dev(finish = false) once the work it enqueued is done: the root, and the error
// of a bounded device wait if one gave up.  Nothing may overwrite the context's tail in between.
void commit_finish(lgs_ctx* c, lgs_commit_data* cd) {
  LGS_CUDA(cudaStreamSynchronize(c->st));
  LGS_CUDA(cudaStreamSynchronize(c->hs));
  c->prof.flush();
  int err = 0;
  std::memcpy(&err, c->tail.as<uint8_t>(), sizeof(int));
  std::memcpy(cd->root.b, c->tail.as<uint8_t>() + 32, 32);
  cd->root_ready = true;
  if (err) {
    LGS_CUDA(cudaMemsetAsync(c->err.p, 0, sizeof(int), c->st));
    LGS_CUDA(cudaStreamSynchronize(c->st));
    throw DeviceTimeout("subset-sum hash: a bounded device wait gave up (code " +
                        std::to_string(err) + ")");
  }
}

// ---------------------------------------------------------------------------------------------
// prove
// ---------------------------------------------------------------------------------------------
namespace {

// Staging buffer layout (u64 offsets) for everything the proof reads back from the device.
struct Stage {
  size_t total = 0;
  size_t take(size_t words) {
    size_t o = total;
    total += words;
    return o;
  }
};

struct SegPlan {
  std::vector<GatherSeg> segs;  // idx and dst hold offsets until relocated
  std::vector<uint64_t> idx;    // all index lists, concatenated
  void add(const u64* src, const std::vector<uint64_t>& items, unsigned words, size_t dst_off) {
    GatherSeg g;
    g.src = src;
    g.idx = (const uint64_t*)(uintptr_t)idx.size();
    g.count = items.size();
    g.words = words;
    g.dst = (u64*)(uintptr_t)dst_off;
    idx.insert(idx.end(), items.begin(), items.end());
    segs.push_back(g);
  }
};

struct OpenPlan {  // one Merkle opening read back from the device
  size_t node_off, nnodes, val_off;
  std::vector<uint64_t> keys;
  unsigned words;
};

const size_t SC_D[7] = {3, 2, 2, 2, 2, 2, 2};

}  // namespace

// The captured prove for this shape, capturing it now if the arena is already sized for it (an
// eager prove of the shape has run); nullptr when this prove must run eagerly.
template <class F>
const ProveGraph* prove_graph(lgs_ctx* c, const Shape& s, F&& enqueue) {
  if (!c->use_graphs) return nullptr;
  ProveGraph* g = nullptr;
  for (auto& e : c->graphs)
    if (e.log_m == s.log_m && e.log_n == s.log_n) g = &e;
  if (!g) {
    c->graphs.emplace_back();
    c->graphs.back().log_m = s.log_m;
    c->graphs.back().log_n = s.log_n;
    return nullptr;
  }
  const Arena& ar = c->arena;
  const bool tl = c->prof_level >= 2;
  if (g->exec && g->arena == ar.mem.p && g->arena_bytes == ar.mem.bytes && g->up == c->up.p &&
      g->down == c->down.p && g->timeline == tl)
    return g;
  if (g->exec) {
    LGS_CUDA(cudaGraphExecDestroy(g->exec));
    g->exec = nullptr;
  }
  if (g->need == 0 || g->need > ar.mem.bytes || !ar.overflow.empty()) return nullptr;
  cudaGraph_t graph = nullptr;
  LGS_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  const uint64_t l0 = thread_launches();
  c->arena.frozen = true;
  try {
    enqueue();
  } catch (...) {
    c->arena.frozen = false;
    cudaStreamEndCapture(c->st, &graph);
    if (graph) cudaGraphDestroy(graph);
    (void)cudaGetLastError();
    throw;
  }
  c->arena.frozen = false;
  const uint64_t captured = thread_launches() - l0;
  adjust_launches(-(int64_t)captured);  // captured, not launched
  LGS_CUDA(cudaStreamEndCapture(c->st, &graph));
  cudaGraphExec_t exec = nullptr;
  // kernel nodes keep the priority of the stream they were captured from
  const cudaError_t err =
      cudaGraphInstantiateWithFlags(&exec, graph, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(graph);
  LGS_CUDA(err);
  g->exec = exec;
  g->timeline = tl;
  g->launches = captured;
  g->arena = ar.mem.p;
  g->arena_bytes = ar.mem.bytes;
  g->up = c->up.p;
  g->down = c->down.p;
  return g;
}

namespace {
thread_local std::function<void(const std::string&, cudaStream_t)>* t_tl_hook = nullptr;
thread_local const char* t_tl_branch = "";
}  // namespace

void tl_mark(const char* what, cudaStream_t st) {
  if (t_tl_hook) (*t_tl_hook)(std::string(t_tl_branch) + "/" + what, st);
}

void note_prove_need(lgs_ctx* c, const Shape& s, size_t need) {
  for (auto& e : c->graphs)
    if (e.log_m == s.log_m && e.log_n == s.log_n) e.need = std::max(e.need, need);
}

void prove_dev(lgs_ctx* c, const lgs_pk* pk, const lgs_commit_data* cd, const u64* z_host,
               size_t zlen, const u64* fields_host, size_t nfields, const uint64_t* ints_host,
               size_t nints, uint64_t cursors[2], std::vector<uint8_t>* proof_out) {
  const Shape& s = pk->shape;
  if (cd->shape.log_m != s.log_m || cd->shape.log_n != s.log_n)
    throw ShapeError("prove: commitment shape differs from the key");
  if (zlen != s.log_m + s.log_n) throw ShapeError("prove: point length must be log_m + log_n");
  const size_t m = s.m(), n = s.n(), two_n = 2 * n, W = s.W(), S = NUM_COLS;
  const unsigned log_n = s.log_n, log_w = s.log_w(), log_s = s.log_s();
  const unsigned nb = log_w + log_s, R = s.R();
  const size_t D = s.D(), WS = W * S;
  const FieldPlan fp(s);
  const uint64_t f0 = cursors[0], i0 = cursors[1];
  if (f0 > nfields || nfields - f0 < fp.total) throw OracleError("oracle exhausted (fields)");
  if (i0 > nints || nints - i0 < INTS_PER_PROOF) throw OracleError("oracle exhausted (ints)");
  cudaStream_t st = c->st;
  Arena& ar = c->arena;
  HostClock hc(c->prof);
  ar.begin();

  // ---- host transcript: indices and points --------------------------------------------------
  std::vector<uint64_t> idx;
  if (!sample_columns(ints_host + i0, two_n, &idx))
    throw OracleError("not enough distinct columns sampled from oracle");
  std::vector<uint64_t> sorted_idx(idx);
  std::sort(sorted_idx.begin(), sorted_idx.end());
  const std::vector<uint64_t> base = query_base(ints_host + i0 + 4 * NUM_COLS, D / 2);
  const std::vector<uint64_t> bpos = level_positions(base, D / 2);

  const u64* F = fields_host + 2 * f0;  // EF fields from the cursor
  auto fld = [&](unsigned off) { return ef_make(F[2 * off], F[2 * off + 1]); };
  auto slice = [&](unsigned off, unsigned len) {
    std::vector<ef2> v(len);
    for (unsigned i = 0; i < len; ++i) v[i] = fld(off + i);
    return v;
  };
  auto rev = [](std::vector<ef2> v) {
    std::reverse(v.begin(), v.end());
    return v;
  };
  auto cat = [](std::vector<ef2> a, const std::vector<ef2>& b) {
    a.insert(a.end(), b.begin(), b.end());
    return a;
  };
  std::vector<ef2> z(zlen);
  for (size_t i = 0; i < zlen; ++i) z[i] = ef_make(gl_canon(z_host[2 * i]), gl_canon(z_host[2 * i + 1]));
  const std::vector<ef2> z2(z.begin(), z.begin() + log_n), z1(z.begin() + log_n, z.end());
  const auto alpha2 = slice(fp.alpha2, 5);
  const auto r2 = slice(fp.r2, log_s);
  const auto r1 = rev(slice(fp.ch_bin, nb));
  const auto r4 = rev(slice(fp.ch_hash, log_w));
  const auto r5 = rev(slice(fp.ch_recon, log_w));
  const auto r3 = rev(slice(fp.ch_table, log_n + 1));
  const auto r6 = rev(slice(fp.ch_rs, log_n));
  const auto r_bi = rev(slice(fp.ch_bi, nb));
  const auto r_a = rev(slice(fp.ch_a, log_n));
  const auto p_a = cat(r4, alpha2);
  const auto p_bi_hash = cat(r2, r4);
  const auto p_bi_recon = cat(r2, r5);

  // ---- parameter block ---------------------------------------------------------------------
  std::vector<ef2> prm;  // EF section
  auto put = [&](const std::vector<ef2>& v) {
    size_t o = prm.size();
    prm.insert(prm.end(), v.begin(), v.end());
    return o;
  };
  const size_t P_fields = put(slice(0, fp.total));
  const size_t P_z1 = put(z1), P_z2 = put(z2), P_r3 = put(r3);
  const size_t P_bipts = put(cat(cat(r1, p_bi_hash), p_bi_recon));
  const size_t P_apts = put(cat(z2, r6));
  const size_t P_pa = put(p_a), P_rbi = put(r_bi), P_ra = put(r_a);
  // batched-open evaluation points Q_{c,t} = (r_0 .. r_{t-1}, 0, zp_c[t+1] .. zp_c[R-1])
  size_t P_q;
  {
    const std::vector<ef2>* cpts[3] = {&p_a, &r_bi, &r_a};
    const unsigned cli[3] = {s.li(s.na()), s.li(s.nbi()), s.li(s.naa())};
    const auto rb = slice(fp.ch_batch, R);
    std::vector<ef2> q;
    for (int ch = 0; ch < 3; ++ch)
      for (unsigned t = 0; t < R; ++t)
        for (unsigned u = 0; u < R; ++u)
          q.push_back(u < t ? rb[u] : (u == t ? ef_zero() : (*cpts[ch])[cli[ch] + u]));
    P_q = put(q);
  }

  // ---- staging layout ----------------------------------------------------------------------
  // Every region is sized by its upper bound for the shape, so offsets (and every kernel
  // argument below) depend on the shape only and a captured graph of the prove replays for any
  // transcript; the transcript-dependent counts travel in the uploaded gather plan.
  Stage sg;
  const size_t S_y = sg.take(2), S_y4 = sg.take(2), S_y5 = sg.take(2);
  const size_t S_coma = sg.take(4), S_comi = sg.take(4);
  const size_t S_hcols = sg.take(S * DIGEST_ROWS);
  const std::vector<uint64_t> h_nodes = multiproof_nodes(sorted_idx, two_n);
  const size_t S_hopen = sg.take(multiproof_bound(S, two_n) * 4);
  const unsigned sc_k[7] = {nb, log_w, log_w, log_n + 1, log_n, nb, log_n};
  size_t S_sc_r[7], S_sc_f[7];
  for (int i = 0; i < 7; ++i) {
    S_sc_r[i] = sg.take(sc_k[i] * (SC_D[i] + 1) * 2);
    S_sc_f[i] = sg.take(SC_D[i] * 2);
  }
  const unsigned NCH = 3;
  const size_t S_msgs = sg.take(NCH * R * 2);
  const size_t S_roots = sg.take((R ? R - 1 : 0) * 4);
  const size_t final_len = D >> R;
  const size_t S_final = sg.take(final_len * 2);
  // Merkle openings: base positions of the three channels, then one per fold level
  const unsigned li_a = s.li(s.naa()), li_bi = s.li(s.nbi()), li_A = s.li(s.na());
  const unsigned chan_li[3] = {li_A, li_bi, li_a};
  const int chan_ef[3] = {0, 0, 1};
  const std::vector<uint64_t> b_nodes = multiproof_nodes(bpos, D);
  size_t idx_bound = S * DIGEST_ROWS + multiproof_bound(S, two_n) + 2 + final_len;
  std::vector<OpenPlan> opens;  // base_bf(A), base_bf(B_I), base_ef(a), then fold levels
  {
    const uint64_t qmax = std::min<uint64_t>(2 * QUERIES, D);  // level_positions(base, D / 2)
    for (int ch = 0; ch < 3; ++ch) {
      OpenPlan o;
      o.nnodes = b_nodes.size();
      o.node_off = sg.take(multiproof_bound(qmax, D) * 4);
      o.words = ((1u << chan_li[ch]) * (chan_ef[ch] ? 2 : 1));
      o.val_off = sg.take(qmax * o.words);
      o.keys = bpos;
      opens.push_back(o);
      idx_bound += multiproof_bound(qmax, D) + qmax;
    }
  }
  std::vector<std::vector<uint64_t>> lvl_pos(R), lvl_mp(R);
  for (unsigned k = 1; k < R; ++k) {
    OpenPlan o;
    const uint64_t len = D >> k, qmax = std::min<uint64_t>(2 * QUERIES, len);
    lvl_pos[k] = level_positions(base, len / 2);
    lvl_mp[k] = multiproof_nodes(lvl_pos[k], len);
    o.nnodes = lvl_mp[k].size();
    o.node_off = sg.take(multiproof_bound(qmax, len) * 4);
    o.words = 2;
    o.val_off = sg.take(qmax * 2);
    o.keys = lvl_pos[k];
    opens.push_back(o);
    idx_bound += multiproof_bound(qmax, len) + qmax + 1;
  }

  // ---- device buffers (arena offsets only: nothing here waits for the device) ----------------
  ef2* eqz1 = ar.get<ef2>(m);
  ef2* a_vec = ar.get<ef2>(n);
  ef2* ra = ar.get<ef2>(two_n);
  BasefoldDev a_st, bi_st;  // Basefold states built during prove
  a_st.codes = ar.get<u64>(D * ((size_t)2 << li_a));
  a_st.nodes = ar.get<u32>((2 * D - 1) * 8);
  bi_st.codes = ar.get<u64>(D * ((size_t)1 << li_bi));
  bi_st.nodes = ar.get<u32>((2 * D - 1) * 8);
  u64* bi = ar.get<u64>(WS);
  u64* stage = ar.get<u64>(sg.total);
  ef2* eq_a2 = ar.get<ef2>(DIGEST_ROWS);
  ef2* eq_r2 = ar.get<ef2>(S);
  ef2* levels = ar.get<ef2>(2 * D);
  std::vector<u32*> lvl_nodes(R, nullptr);
  for (unsigned k = 1; k < R; ++k) lvl_nodes[k] = ar.get<u32>((2 * (D >> k) - 1) * 8);
  const size_t mlen = (size_t)1 << R;
  ef2* mch[3];
  for (int ch = 0; ch < 3; ++ch) mch[ch] = ar.get<ef2>(mlen);
  const BasefoldDev* chan_states[3] = {&pk->a_state, &bi_st, &a_st};
  const u64* polys[3] = {pk->A.as<u64>(), bi, (const u64*)a_vec};

  // ---- the gather plan into staging (pcs/src/ligesis.rs:527-549 fields of the proof) --------
  SegPlan plan;
  {
    std::vector<uint64_t> hidx;  // H[r][sorted_idx[k]], column by column
    hidx.reserve(S * DIGEST_ROWS);
    for (uint64_t j : sorted_idx)
      for (unsigned r = 0; r < DIGEST_ROWS; ++r) hidx.push_back((uint64_t)r * two_n + j);
    plan.add(cd->H.as<u64>(), hidx, 1, S_hcols);
    plan.add((const u64*)cd->nodes.as<u32>(), h_nodes, 4, S_hopen);
    plan.add((const u64*)a_st.nodes, {2 * D - 2}, 4, S_coma);
    plan.add((const u64*)bi_st.nodes, {2 * D - 2}, 4, S_comi);
    for (int ch = 0; ch < 3; ++ch) {
      const OpenPlan& o = opens[ch];
      plan.add((const u64*)chan_states[ch]->nodes, b_nodes, 4, o.node_off);
      plan.add(chan_states[ch]->codes, bpos, o.words, o.val_off);
    }
    size_t off = D;
    for (unsigned k = 1; k < R; ++k) {
      const OpenPlan& o = opens[2 + k];
      const size_t len = D >> k;
      plan.add((const u64*)lvl_nodes[k], lvl_mp[k], 4, o.node_off);
      plan.add((const u64*)(levels + off), lvl_pos[k], 2, o.val_off);
      plan.add((const u64*)lvl_nodes[k], {2 * len - 2}, 4, S_roots + (k - 1) * 4);
      off += len;
    }
    std::vector<uint64_t> fin(final_len);
    for (size_t i = 0; i < final_len; ++i) fin[i] = i;
    plan.add((const u64*)(levels + off), fin, 2, S_final);
  }

  // ---- one upload: parameters, column indices, message tasks, channels, gather plan ---------
  size_t blob = 0;
  auto part = [&](size_t bytes) {
    const size_t o = blob;
    blob += (bytes + 255) & ~(size_t)255;
    return o;
  };
  const size_t U_prm = part(prm.size() * sizeof(ef2));
  const size_t U_idx = part(S * 8);
  const size_t U_tasks = part(3 * R * sizeof(EqDotTask));
  const size_t U_chs = part(3 * sizeof(BfChannelDev));
  // source addresses read by kernels through device slots: f, F', A, B_I, a-bar
  enum { PT_F, PT_CW, PT_A, PT_BI, PT_AVEC, PT_N };
  const size_t U_ptrs = part(PT_N * sizeof(void*));
  if (plan.idx.size() > idx_bound) throw std::logic_error("prove: gather plan exceeds its bound");
  const size_t U_gidx = part(idx_bound * 8);
  const size_t U_segs = part(plan.segs.size() * sizeof(GatherSeg));
  uint8_t* d_up = ar.get<uint8_t>(blob);
  c->up.reserve(blob);
  uint8_t* h_up = c->up.as<uint8_t>();
  const ef2* d_prm = (const ef2*)(d_up + U_prm);
  const ef2* d_fields = d_prm + P_fields;
  const uint64_t* d_idx = (const uint64_t*)(d_up + U_idx);
  const ef2* pts[3] = {d_prm + P_pa, d_prm + P_rbi, d_prm + P_ra};
  std::memcpy(h_up + U_prm, prm.data(), prm.size() * sizeof(ef2));
  std::memcpy(h_up + U_idx, idx.data(), S * 8);
  const u64* const* d_ptrs = (const u64* const*)(d_up + U_ptrs);
  {
    const u64* pt[PT_N] = {cd->fdev(), cd->cw.as<u64>(), pk->A.as<u64>(), bi,
                           (const u64*)a_vec};
    std::memcpy(h_up + U_ptrs, pt, sizeof(pt));
  }
  {
    EqDotTask* tasks = (EqDotTask*)(h_up + U_tasks);
    for (int ch = 0; ch < 3; ++ch)
      for (unsigned t = 0; t < R; ++t) {
        EqDotTask& tk = tasks[ch * R + t];
        tk.vec = mch[ch];
        tk.point = d_prm + P_q + (size_t)(ch * R + t) * R;
        tk.out = (ef2*)(stage + S_msgs) + ch * R + t;
      }
    BfChannelDev* chs = (BfChannelDev*)(h_up + U_chs);
    for (int ch = 0; ch < 3; ++ch) {
      chs[ch].codes = chan_states[ch]->codes;
      chs[ch].poly = polys[ch];
      chs[ch].is_ef = chan_ef[ch];
      chs[ch].li = chan_li[ch];
      chs[ch].point = pts[ch];
    }
    std::memcpy(h_up + U_gidx, plan.idx.data(), plan.idx.size() * 8);
    GatherSeg* segs = (GatherSeg*)(h_up + U_segs);
    for (size_t i = 0; i < plan.segs.size(); ++i) {
      segs[i] = plan.segs[i];
      segs[i].idx = (const uint64_t*)(d_up + U_gidx) + (uintptr_t)plan.segs[i].idx;
      segs[i].dst = stage + (uintptr_t)plan.segs[i].dst;
    }
  }
  c->down.reserve(sg.total * 8);

  hc.lap("host_plan");

  // Everything from the upload to the read-back depends on the transcript only through the
  // uploaded blob, so it is captured once per shape into a CUDA graph and replayed.
  const bool tl = c->prof_level >= 2;
  unsigned ntl = 0;
  if (tl)
    for (int i = 0; i < lgs_ctx::TL_MAX; ++i)
      if (!c->tl_ev[i]) LGS_CUDA(cudaEventCreate(&c->tl_ev[i]));
  auto mark = [&](const std::string& name, cudaStream_t where) {
    if (!tl || ntl >= (unsigned)lgs_ctx::TL_MAX) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    LGS_CUDA(cudaStreamIsCapturing(where, &cs));
    if (cs == cudaStreamCaptureStatusActive)
      LGS_CUDA(cudaEventRecordWithFlags(c->tl_ev[ntl], where, cudaEventRecordExternal));
    else
      LGS_CUDA(cudaEventRecord(c->tl_ev[ntl], where));
    if (c->tl_names.size() <= ntl) c->tl_names.resize(ntl + 1);
    c->tl_names[ntl++] = name;
  };
  std::function<void(const std::string&, cudaStream_t)> hook = mark;
  struct HookScope {  // tl_mark() reaches `mark` only while this prove is enqueued
    HookScope(std::function<void(const std::string&, cudaStream_t)>* h, bool on) {
      t_tl_hook = on ? h : nullptr;
      t_tl_branch = "";
    }
    ~HookScope() { t_tl_hook = nullptr; }
  };
  auto enqueue = [&]() {
  HookScope hook_scope(&hook, tl);
  ntl = 0;
  mark("start", st);
  h2d(d_up, h_up, blob, st);

  // -- the transcript is a DAG of independent branches (every challenge is pre-drawn): fork them
  // onto side streams as soon as their inputs exist, join before the gather.  The branches that
  // need only B_I fork before the a-bar GEMV; the two Basefold commitments (A1, B) gate the
  // Stage B codeword chain on the main stream and run on high-priority streams.
  new_eq_dev(d_prm + P_z1, s.log_m, eqz1, st);
  bits_gather(d_ptrs + PT_CW, two_n, d_idx, S, W, bi, st);
  new_eq_dev(d_fields + fp.alpha2, 5, eq_a2, st);
  new_eq_dev(d_fields + fp.r2, log_s, eq_r2, st);
  mark("prefix_end", st);
  LGS_CUDA(cudaEventRecord(c->ev_fork, st));
  std::vector<cudaStream_t> brs;
  unsigned n_hi = 0;
  cudaEvent_t fork_ev = c->ev_fork;
  auto branch = [&](bool hi = false) {
    if (brs.size() >= (size_t)lgs_ctx::NSIDE) throw std::runtime_error("prove: too many branches");
    cudaStream_t b;
    if (hi) {
      if (n_hi >= (unsigned)lgs_ctx::NSIDE_HI) throw std::runtime_error("prove: too many branches");
      b = c->side_hi[n_hi++];
    } else {
      b = c->side[brs.size() - n_hi];
    }
    brs.push_back(b);
    LGS_CUDA(cudaStreamWaitEvent(b, fork_ev, 0));
    return b;
  };
  auto partials_for = [&](unsigned k, unsigned d) {
    return ar.get<ef2>(std::max(sumcheck_partials_elems(k, d), eqdot_partials_elems(k) + 1024));
  };
  const unsigned br_b = (unsigned)brs.size();
  // B: the Basefold commitment to B_I (pcs/src/ligesis.rs:411-416)
  {
    t_tl_branch = "B";
    cudaStream_t b = branch(true);
    bf_commit(c, bi, 0, WS, li_bi, CODE_RATE, &bi_st, b);
    mark("B_bi_commit_end", b);
  }
  // C: binary check, factors [B_I, B_I - 1, eq_alpha1] (pcs/src/ligesis.rs:419-429); the
  // longest branch, so it is the third high-priority one
  {
    t_tl_branch = "C";
    cudaStream_t b = branch(true);
    ef2* p0 = ar.get<ef2>(WS);
    ef2* p2 = ar.get<ef2>(WS);
    lift_bf(bi, p0, WS, 0, b);
    new_eq_dev(d_fields + fp.alpha1, nb, p2, b);
    tl_mark("inputs_end", b);
    sumcheck_binary_dev(p0, p2, nb, d_fields + fp.ch_bin, (ef2*)(stage + S_sc_r[0]),
                        (ef2*)(stage + S_sc_f[0]), partials_for(nb, 3), b, c->sumcheck_blocks);
    mark("C_binary_sc_end", b);
  }
  // D: hash and recon bilinear sumchecks (pcs/src/ligesis.rs:435-485)
  {
    t_tl_branch = "D";
    cudaStream_t b = branch();
    ef2* g1 = ar.get<ef2>(W);
    ef2* g2 = ar.get<ef2>(W);
    ef2* g2b = ar.get<ef2>(W);
    ef2* v = ar.get<ef2>(W);
    g1_build(d_ptrs + PT_A, W, eq_a2, DIGEST_ROWS, g1, b);
    g2_build(bi, W, S, eq_r2, g2, b);
    d2d(g2b, g2, W * sizeof(ef2), b);
    v_build(eqz1, W, v, b);
    tl_mark("inputs_end", b);
    ef2* ph[2] = {g1, g2};
    ef2* part = partials_for(log_w, 2);
    sumcheck_prove_dev(ph, 2, log_w, d_fields + fp.ch_hash, (ef2*)(stage + S_sc_r[1]),
                       (ef2*)(stage + S_sc_f[1]), part, b, c->sumcheck_blocks);
    ef2* pr[2] = {v, g2b};
    sumcheck_prove_dev(pr, 2, log_w, d_fields + fp.ch_recon, (ef2*)(stage + S_sc_r[2]),
                       (ef2*)(stage + S_sc_f[2]), part, b, c->sumcheck_blocks);
    mark("D_hash_recon_sc_end", b);
  }
  // F: Stage A point reduction of B_I (pcs/src/ligesis.rs:510-516)
  {
    t_tl_branch = "F";
    cudaStream_t b = branch();
    ef2* gbi = ar.get<ef2>(WS);
    ef2* bie = ar.get<ef2>(WS);
    combine_eq_dev(d_prm + P_bipts, 3, nb, d_fields + fp.gamma_bi, gbi, b);
    lift_bf(bi, bie, WS, 0, b);
    tl_mark("inputs_end", b);
    ef2* pb[2] = {bie, gbi};
    sumcheck_prove_dev(pb, 2, nb, d_fields + fp.ch_bi, (ef2*)(stage + S_sc_r[5]),
                       (ef2*)(stage + S_sc_f[5]), partials_for(nb, 2), b, c->sumcheck_blocks);
    mark("F_bi_batch_sc_end", b);
  }
  // -- a-bar = eq_{z1}^T F and everything that needs it (pcs/src/ligesis.rs:365-387)
  gemv_eq_rows(d_ptrs + PT_F, eqz1, m, n, a_vec, st);
  mark("abar_end", st);
  LGS_CUDA(cudaEventRecord(c->ev_fork2, st));
  fork_ev = c->ev_fork2;
  const unsigned br_a1 = (unsigned)brs.size();
  // A1: y = a(z2) and the Basefold commitment to a-bar (pcs/src/ligesis.rs:379-384)
  {
    t_tl_branch = "A1";
    cudaStream_t b = branch(true);
    eq_dot_dev(a_vec, 0, d_prm + P_z2, log_n, (ef2*)(stage + S_y), partials_for(log_n, 1), b);
    bf_commit(c, (const u64*)a_vec, 1, n, li_a, CODE_RATE, &a_st, b);
    mark("A1_abar_commit_end", b);
  }
  // A2: RS(a-bar), y4, the recon table sumcheck and y5 (pcs/src/ligesis.rs:387, 458, 487-497)
  {
    t_tl_branch = "A2";
    cudaStream_t b = branch();
    u64* t1 = ar.get<u64>(2 * n);
    u64* t2 = ar.get<u64>(2 * two_n);
    u64* scr = ilog2(two_n) > 12 ? ar.get<u64>(2 * two_n) : nullptr;
    transpose_u64((const u64*)a_vec, t1, n, 2, 1, b);
    ntt_batch(t1, n, n, t2, two_n, ilog2(two_n), 2, scr, c->tw.as<u64>(), b);
    transpose_u64(t2, (u64*)ra, 2, two_n, 1, b);
    tl_mark("rs_end", b);
    y4_dev(eq_r2, ra, d_idx, S, (ef2*)(stage + S_y4), b);
    ef2* sel = ar.get<ef2>(two_n);
    ef2* rac = ar.get<ef2>(two_n);
    sel_build(d_idx, eq_r2, S, two_n, sel, b);
    d2d(rac, ra, two_n * sizeof(ef2), b);
    ef2* pt[2] = {sel, rac};
    sumcheck_prove_dev(pt, 2, log_n + 1, d_fields + fp.ch_table, (ef2*)(stage + S_sc_r[3]),
                       (ef2*)(stage + S_sc_f[3]), partials_for(log_n + 1, 2), b, c->sumcheck_blocks);
    eq_dot_dev(ra, 0, d_prm + P_r3, log_n + 1, (ef2*)(stage + S_y5), partials_for(log_n + 1, 1), b);
    mark("A2_rs_abar_table_sc_end", b);
  }
  // E: RS-link sumcheck (pcs/src/ligesis.rs:499-502); r3 is pre-drawn, so w needs no wait
  {
    t_tl_branch = "E";
    cudaStream_t b = branch();
    ef2* w = ar.get<ef2>(n);
    ef2* ac = ar.get<ef2>(n);
    rs_weights_dev(d_prm + P_r3, log_n + 1, n, c->tw.as<u64>(), w, b);
    d2d(ac, a_vec, n * sizeof(ef2), b);
    ef2* pw[2] = {ac, w};
    sumcheck_prove_dev(pw, 2, log_n, d_fields + fp.ch_rs, (ef2*)(stage + S_sc_r[4]),
                       (ef2*)(stage + S_sc_f[4]), partials_for(log_n, 2), b, c->sumcheck_blocks);
    mark("E_rslink_sc_end", b);
  }
  // G: Stage A point reduction of a-bar (pcs/src/ligesis.rs:518-522)
  {
    t_tl_branch = "G";
    cudaStream_t b = branch();
    ef2* ga = ar.get<ef2>(n);
    ef2* ac = ar.get<ef2>(n);
    combine_eq_dev(d_prm + P_apts, 2, log_n, d_fields + fp.gamma_a, ga, b);
    d2d(ac, a_vec, n * sizeof(ef2), b);
    ef2* pa[2] = {ac, ga};
    sumcheck_prove_dev(pa, 2, log_n, d_fields + fp.ch_a, (ef2*)(stage + S_sc_r[6]),
                       (ef2*)(stage + S_sc_f[6]), partials_for(log_n, 2), b, c->sumcheck_blocks);
    mark("G_a_batch_sc_end", b);
  }
  // H: Stage B reduction messages (pcs/src/basefold.rs:746-769).  With m = poly.fold(point[0..li])
  // (2^R values) and the batch challenges r_0.., round t's l0 = MLE(m)(r_0, .., r_{t-1}, 0,
  // zp[t+1], .., zp[R-1]): the sequential rounds collapse to R independent evaluations.
  {
    t_tl_branch = "H";
    cudaStream_t b = branch();
    const int poly_slot[3] = {PT_A, PT_BI, PT_AVEC};
    for (int ch = 0; ch < 3; ++ch)
      bf_fold_poly_dev(d_ptrs + poly_slot[ch], chan_ef[ch], chan_li[ch], pts[ch], mlen, mch[ch], b);
    ef2* part = ar.get<ef2>(eq_dot_multi_partials(R, 3 * R));
    eq_dot_multi_dev((const EqDotTask*)(d_up + U_tasks), 3 * R, R, part, b);
    mark("H_basefold_msgs_end", b);
  }
  t_tl_branch = "main";
  // join: main waits for every branch
  for (size_t i = 0; i < brs.size(); ++i) LGS_CUDA(cudaEventRecord(c->ev_done[i], brs[i]));
  LGS_CUDA(cudaStreamWaitEvent(st, c->ev_done[br_a1], 0));
  LGS_CUDA(cudaStreamWaitEvent(st, c->ev_done[br_b], 0));
  mark("main_suffix_start", st);
  // Stage B codeword chain on main (needs both prove-time commitments): combined level 0,
  // the R folds, and the Merkle trees of levels 1..R-1 (pcs/src/basefold.rs:735-784)
  bf_combine_dev((const BfChannelDev*)(d_up + U_chs), 3, d_fields + fp.coeffs, D, levels, st);
  bf_levels_dev(levels, D, R, d_fields + fp.ch_batch, c->tw.as<u64>(), st);
  mark("main_levels_end", st);
  if (R > 1) {
    std::vector<const u64*> ldata;
    std::vector<u32*> lnodes;
    std::vector<size_t> lcount;
    size_t off = D;
    for (unsigned k = 1; k < R; ++k) {
      const size_t len = D >> k;
      ldata.push_back((const u64*)(levels + off));
      lnodes.push_back(lvl_nodes[k]);
      lcount.push_back(len);
      off += len;
    }
    merkle_leaves_many(ldata.data(), 2, lnodes.data(), lcount.data(), (unsigned)lnodes.size(), st);
    merkle_build_many(lnodes.data(), lcount.data(), (unsigned)lnodes.size(), st);
  }
  mark("main_level_trees_end", st);
  for (size_t i = 0; i < brs.size(); ++i) LGS_CUDA(cudaStreamWaitEvent(st, c->ev_done[i], 0));
  mark("join", st);
  c->tl_count = ntl;
  };
  const ProveGraph* graph = prove_graph(c, s, enqueue);
  StageTimer t_prove(c->prof, st, "prove_device");
  if (graph) {
    LGS_CUDA(cudaGraphLaunch(graph->exec, st));
    adjust_launches((int64_t)graph->launches);
  } else {
    enqueue();
    note_prove_need(c, s, ar.off);
  }
  ntl = c->tl_count;
  // ---- gathers into staging, one read-back: after the commitment's tree (the only thing the
  // prove reads from the commit's hash stream: H columns and their Merkle nodes) -------------
  if (cd->done) LGS_CUDA(cudaStreamWaitEvent(st, cd->done, 0));
  mark("tree_ready", st);
  gather_segments((const GatherSeg*)(d_up + U_segs), (unsigned)plan.segs.size(), st);
  LGS_CUDA(cudaMemcpyAsync(c->down.p, stage, sg.total * 8, cudaMemcpyDeviceToHost, st));
  mark("end", st);
  t_prove.stop();
  hc.lap("host_enqueue");
  const u64* hst = c->down.as<u64>();
  LGS_CUDA(cudaStreamSynchronize(st));
  hc.lap("host_wait");
  c->prof.flush();
  if (tl && c->tl_ev[0]) {
    for (unsigned i = 1; i < c->tl_names.size() && i < (unsigned)lgs_ctx::TL_MAX; ++i) {
      float ms = 0;
      if (c->tl_ev[i] && cudaEventElapsedTime(&ms, c->tl_ev[0], c->tl_ev[i]) == cudaSuccess)
        c->prof.add("tl:" + c->tl_names[i], ms);
    }
  }

  // ---- encode straight from the staging buffer, in the order of encode_proof --------------
  ByteWriter w(*proof_out);
  w.need(sg.total * 8 + 4096);
  w.raw("LGSP", 4);
  w.u32v(1);
  w.bf_run(hst + S_y, 2);
  w.raw(hst + S_coma, 32);
  w.raw(hst + S_comi, 32);
  w.bf_run(hst + S_y4, 2);
  w.bf_run(hst + S_y5, 2);
  w.u32v((uint32_t)S);
  w.u32v(DIGEST_ROWS);
  w.bf_run(hst + S_hcols, S * DIGEST_ROWS);
  w.u32v((uint32_t)(h_nodes.size() * 32));
  w.raw(hst + S_hopen, h_nodes.size() * 32);
  for (int i = 0; i < 7; ++i) {  // ScProof: rounds, width, round values, finals
    w.u32v(sc_k[i]);
    w.u32v(sc_k[i] ? (uint32_t)(SC_D[i] + 1) : 0);
    w.bf_run(hst + S_sc_r[i], (size_t)sc_k[i] * (SC_D[i] + 1) * 2);
    w.u32v((uint32_t)SC_D[i]);
    w.bf_run(hst + S_sc_f[i], SC_D[i] * 2);
  }
  w.u32v(CODE_RATE);
  w.u32v(ilog2(D));
  w.u32v(NCH);
  for (unsigned ch = 0; ch < NCH; ++ch) {
    w.u32v(R);
    w.bf_run(hst + S_msgs + (size_t)ch * R * 2, (size_t)R * 2);
  }
  w.u32v(R ? R - 1 : 0);
  if (R > 1) w.raw(hst + S_roots, (size_t)(R - 1) * 32);
  w.u32v((uint32_t)final_len);
  w.bf_run(hst + S_final, final_len * 2);
  auto opening = [&](const OpenPlan& o, bool ef) {  // Merkle bytes, then (key, values) pairs
    w.u32v((uint32_t)(o.nnodes * 32));
    w.raw(hst + o.node_off, o.nnodes * 32);
    w.u32v((uint32_t)o.keys.size());
    for (size_t i = 0; i < o.keys.size(); ++i) {
      w.u64v(o.keys[i]);
      w.u32v(ef ? o.words / 2 : o.words);
      w.bf_run(hst + o.val_off + i * o.words, o.words);
    }
  };
  w.u32v(R ? R - 1 : 0);  // fold openings
  for (size_t oi = 3; oi < opens.size(); ++oi) opening(opens[oi], true);
  w.u32v(2);  // base_bf: A, B_I
  opening(opens[0], false);
  opening(opens[1], false);
  w.u32v(1);  // base_ef: a-bar
  opening(opens[2], true);
  w.finish_in_place();
  hc.lap("host_assemble");
  cursors[0] = f0 + fp.total;
  cursors[1] = i0 + INTS_PER_PROOF;
}

// ---------------------------------------------------------------------------------------------
// standalone Basefold (pcs/src/basefold.rs:309-516)
// ---------------------------------------------------------------------------------------------
void basefold_commit_dev(lgs_ctx* c, const u64* poly, size_t len, int is_ef, unsigned code_rate,
                         unsigned li, lgs_basefold* out) {
  if (len < 2 || (len & (len - 1))) throw ShapeError("basefold: 2^n values, n >= 1");
  const unsigned n = ilog2(len);
  if (li > LOG_INTERLEAVE || li >= n) throw ShapeError("basefold: 0 <= log_interleave < n, <= 6");
  if (code_rate < 1 || n - li + code_rate > TW_LOG)
    throw ShapeError("basefold: code_rate >= 1 and a code length up to 2^22");
  const size_t words = len * (is_ef ? 2 : 1);
  const size_t L = (len >> li) << code_rate;
  const size_t cols = ((size_t)1 << li) * (is_ef ? 2 : 1);
  out->device = c->device;
  out->code_rate = code_rate;
  c->arena.begin();
  out->poly.alloc(words * 8, c->st);
  out->codes.alloc(L * cols * 8, c->st);
  out->nodes.alloc((2 * L - 1) * 32, c->st);
  for (DevMem* d : {&out->poly, &out->codes, &out->nodes}) d->detach(release_stream(c->device));
  h2d_staged(c, out->poly.p, poly, words * 8, c->st);
  canon_u64(out->poly.as<u64>(), words, c->st);
  out->st.codes = out->codes.as<u64>();
  out->st.nodes = out->nodes.as<u32>();
  bf_commit(c, out->poly.as<u64>(), is_ef, len, li, code_rate, &out->st, c->st);
  LGS_CUDA(cudaMemcpyAsync(out->root.b, out->nodes.as<u32>() + (2 * L - 2) * 8, 32,
                           cudaMemcpyDeviceToHost, c->st));
  LGS_CUDA(cudaStreamSynchronize(c->st));
}

void basefold_prove_dev(lgs_ctx* c, const lgs_basefold* bf, const u64* point_host, size_t plen,
                        const u64* fields_host, size_t nfields, const uint64_t* ints_host,
                        size_t nints, uint64_t cursors[2], std::vector<uint8_t>* proof_out) {
  const BasefoldDev& B = bf->st;
  const unsigned n = B.num_vars, li = B.li, R = n - li, cr = bf->code_rate;
  const size_t L = B.L, final_len = L >> R, q = (100 + cr - 1) / cr;  // query_num, :107-109
  const unsigned words = B.leaf_words();
  if (plen != n) throw ShapeError("basefold prove: the point must have num_vars coordinates");
  const uint64_t f0 = cursors[0], i0 = cursors[1];
  if (f0 > nfields || nfields - f0 < R) throw OracleError("oracle exhausted (fields)");
  if (i0 > nints || nints - i0 < q) throw OracleError("oracle exhausted (ints)");
  cudaStream_t st = c->st;
  Arena& ar = c->arena;
  ar.begin();

  // ---- host transcript ------------------------------------------------------------------
  std::vector<ef2> pt(n), rch(R);
  for (unsigned i = 0; i < n; ++i)
    pt[i] = ef_make(gl_canon(point_host[2 * i]), gl_canon(point_host[2 * i + 1]));
  for (unsigned t = 0; t < R; ++t)
    rch[t] = ef_make(fields_host[2 * (f0 + t)], fields_host[2 * (f0 + t) + 1]);
  std::vector<uint64_t> base;  // q ints mod L/2, sorted and deduplicated (:787-795)
  for (size_t t = 0; t < q; ++t) base.push_back(ints_host[i0 + t] % (L / 2));
  std::sort(base.begin(), base.end());
  base.erase(std::unique(base.begin(), base.end()), base.end());
  const std::vector<uint64_t> bpos = level_positions(base, L / 2);
  const std::vector<uint64_t> b_nodes = multiproof_nodes(bpos, L);
  std::vector<std::vector<uint64_t>> lvl_pos(R), lvl_mp(R);
  for (unsigned k = 1; k < R; ++k) {
    lvl_pos[k] = level_positions(base, (L >> k) / 2);
    lvl_mp[k] = multiproof_nodes(lvl_pos[k], L >> k);
  }
  // round t's messages are MLE(m) at (r_0 .. r_{t-1}, b, zp[t+1] .. zp[R-1]), b = 0, 1, with
  // m = poly.fold(point[0..li]) (the reference folds m round by round, :419-443)
  std::vector<ef2> qpts;
  for (unsigned t = 0; t < R; ++t)
    for (unsigned bit = 0; bit < 2; ++bit)
      for (unsigned u = 0; u < R; ++u)
        qpts.push_back(u < t ? rch[u] : (u == t ? (bit ? ef_one() : ef_zero()) : pt[li + u]));

  // ---- staging layout (exact: this prove runs eagerly) --------------------------------------
  Stage sg;
  const size_t S_y = sg.take(2), S_msgs = sg.take((size_t)R * 4);
  const size_t S_roots = sg.take((size_t)(R - 1) * 4), S_final = sg.take(final_len * 2);
  const size_t S_bnodes = sg.take(b_nodes.size() * 4), S_bvals = sg.take(bpos.size() * words);
  std::vector<size_t> S_lnodes(R), S_lvals(R);
  for (unsigned k = 1; k < R; ++k) {
    S_lnodes[k] = sg.take(lvl_mp[k].size() * 4);
    S_lvals[k] = sg.take(lvl_pos[k].size() * 2);
  }

  // ---- device buffers --------------------------------------------------------------------
  ef2* levels = ar.get<ef2>(2 * L);
  std::vector<u32*> lvl_nodes(R, nullptr);
  for (unsigned k = 1; k < R; ++k) lvl_nodes[k] = ar.get<u32>((2 * (L >> k) - 1) * 8);
  const size_t mlen = (size_t)1 << R;
  ef2* mv = ar.get<ef2>(mlen);
  ef2* part1 = ar.get<ef2>(eqdot_partials_elems(n) + 1024);
  ef2* part2 = ar.get<ef2>(eq_dot_multi_partials(R, 2 * R));
  u64* stage = ar.get<u64>(sg.total);

  SegPlan plan;
  plan.add((const u64*)B.nodes, b_nodes, 4, S_bnodes);
  plan.add(B.codes, bpos, words, S_bvals);
  {
    size_t off = L;
    for (unsigned k = 1; k < R; ++k) {
      const size_t len = L >> k;
      plan.add((const u64*)lvl_nodes[k], lvl_mp[k], 4, S_lnodes[k]);
      plan.add((const u64*)(levels + off), lvl_pos[k], 2, S_lvals[k]);
      plan.add((const u64*)lvl_nodes[k], {2 * len - 2}, 4, S_roots + (k - 1) * 4);
      off += len;
    }
    std::vector<uint64_t> fin(final_len);
    for (size_t i = 0; i < final_len; ++i) fin[i] = i;
    plan.add((const u64*)(levels + off), fin, 2, S_final);
  }

  // ---- one upload: point, challenges, message points, one-channel table, pointer, plan -------
  size_t blob = 0;
  auto part = [&](size_t bytes) {
    const size_t o = blob;
    blob += (bytes + 255) & ~(size_t)255;
    return o;
  };
  const size_t U_pt = part(n * sizeof(ef2)), U_ch = part(R * sizeof(ef2));
  const size_t U_q = part(qpts.size() * sizeof(ef2)), U_one = part(sizeof(ef2));
  const size_t U_tasks = part(2 * R * sizeof(EqDotTask)), U_chs = part(sizeof(BfChannelDev));
  const size_t U_ptr = part(sizeof(void*)), U_gidx = part(plan.idx.size() * 8);
  const size_t U_segs = part(plan.segs.size() * sizeof(GatherSeg));
  uint8_t* d_up = ar.get<uint8_t>(blob);
  c->up.reserve(blob);
  uint8_t* h_up = c->up.as<uint8_t>();
  std::memcpy(h_up + U_pt, pt.data(), n * sizeof(ef2));
  std::memcpy(h_up + U_ch, rch.data(), R * sizeof(ef2));
  std::memcpy(h_up + U_q, qpts.data(), qpts.size() * sizeof(ef2));
  const ef2 one = ef_one();
  std::memcpy(h_up + U_one, &one, sizeof(ef2));
  const ef2* d_pt = (const ef2*)(d_up + U_pt);
  {
    EqDotTask* tasks = (EqDotTask*)(h_up + U_tasks);
    for (unsigned i = 0; i < 2 * R; ++i) {
      tasks[i].vec = mv;
      tasks[i].point = (const ef2*)(d_up + U_q) + (size_t)i * R;
      tasks[i].out = (ef2*)(stage + S_msgs) + i;
    }
    BfChannelDev* ch = (BfChannelDev*)(h_up + U_chs);
    ch->codes = B.codes;
    ch->poly = bf->poly.as<u64>();
    ch->is_ef = B.is_ef;
    ch->li = li;
    ch->point = d_pt;
    const u64* pp = bf->poly.as<u64>();
    std::memcpy(h_up + U_ptr, &pp, sizeof(pp));
    std::memcpy(h_up + U_gidx, plan.idx.data(), plan.idx.size() * 8);
    GatherSeg* segs = (GatherSeg*)(h_up + U_segs);
    for (size_t i = 0; i < plan.segs.size(); ++i) {
      segs[i] = plan.segs[i];
      segs[i].idx = (const uint64_t*)(d_up + U_gidx) + (uintptr_t)plan.segs[i].idx;
      segs[i].dst = stage + (uintptr_t)plan.segs[i].dst;
    }
  }
  c->down.reserve(sg.total * 8);

  // ---- device dataflow (pcs/src/basefold.rs:398-476) ----------------------------------------
  h2d(d_up, h_up, blob, st);
  eq_dot_dev(bf->poly.as<u64>(), B.is_ef ? 0 : 1, d_pt, n, (ef2*)(stage + S_y), part1, st);
  bf_combine_dev((const BfChannelDev*)(d_up + U_chs), 1, (const ef2*)(d_up + U_one), L, levels,
                 st);
  bf_fold_poly_dev((const u64* const*)(d_up + U_ptr), B.is_ef, li, d_pt, mlen, mv, st);
  eq_dot_multi_dev((const EqDotTask*)(d_up + U_tasks), 2 * R, R, part2, st);
  bf_levels_dev(levels, L, R, (const ef2*)(d_up + U_ch), c->tw.as<u64>(), st);
  {
    std::vector<const u64*> ldata;
    std::vector<u32*> lnodes;
    std::vector<size_t> lcount;
    size_t off = L;
    for (unsigned k = 1; k < R; ++k) {
      ldata.push_back((const u64*)(levels + off));
      lnodes.push_back(lvl_nodes[k]);
      lcount.push_back(L >> k);
      off += L >> k;
    }
    for (size_t i = 0; i < lnodes.size(); i += 16) {  // the batched tree kernels take 16 trees
      const unsigned cnt = (unsigned)std::min<size_t>(16, lnodes.size() - i);
      merkle_leaves_many(ldata.data() + i, 2, lnodes.data() + i, lcount.data() + i, cnt, st);
      merkle_build_many(lnodes.data() + i, lcount.data() + i, cnt, st);
    }
  }
  gather_segments((const GatherSeg*)(d_up + U_segs), (unsigned)plan.segs.size(), st);
  LGS_CUDA(cudaMemcpyAsync(c->down.p, stage, sg.total * 8, cudaMemcpyDeviceToHost, st));
  LGS_CUDA(cudaStreamSynchronize(st));
  const u64* hst = c->down.as<u64>();

  // ---- encode ("LGSB", proof.hpp) ----------------------------------------------------------
  ByteWriter w(*proof_out);
  w.need(sg.total * 8 + 4096);
  w.raw("LGSB", 4);
  w.u32v(1);
  w.u32v(n);
  w.u32v(cr);
  w.u32v(li);
  w.u32v(B.is_ef ? 1 : 0);
  w.bf_run(hst + S_y, 2);
  w.u32v(R);
  w.bf_run(hst + S_msgs, (size_t)R * 4);
  w.u32v(R - 1);
  w.raw(hst + S_roots, (size_t)(R - 1) * 32);
  w.u32v((uint32_t)final_len);
  w.bf_run(hst + S_final, final_len * 2);
  auto opening = [&](size_t node_off, size_t nnodes, const std::vector<uint64_t>& keys,
                     size_t val_off, unsigned vwords, unsigned nvals) {
    w.u32v((uint32_t)(nnodes * 32));
    w.raw(hst + node_off, nnodes * 32);
    w.u32v((uint32_t)keys.size());
    for (size_t i = 0; i < keys.size(); ++i) {
      w.u64v(keys[i]);
      w.u32v(nvals);
      w.bf_run(hst + val_off + i * vwords, vwords);
    }
  };
  opening(S_bnodes, b_nodes.size(), bpos, S_bvals, words, 1u << li);
  w.u32v(R - 1);
  for (unsigned k = 1; k < R; ++k)
    opening(S_lnodes[k], lvl_mp[k].size(), lvl_pos[k], S_lvals[k], 2, 1);
  w.finish_in_place();
  cursors[0] = f0 + R;
  cursors[1] = i0 + q;
}

}  // namespace lgs
