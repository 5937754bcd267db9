// Host-side state of the prover library: device buffers, the per-context arena, the proving
// key and commitment data (the reference's ProvingKey / CommitData, pcs/src/ligesis.rs:67-97)
// kept resident on the device.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "proof.hpp"

namespace lgs {

// Device buffer from the device's stream-ordered memory pool (cudaMallocAsync on the owning
// context's stream).  The pool keeps freed memory cached (the context raises its release
// threshold), so a commitment allocated and freed per proof costs no cudaMalloc / device sync.
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

// Bump allocator for per-call device scratch.  A call that outgrows the buffer takes extra
// pool allocations; the next call starts from one buffer of the largest size seen, so
// steady-state calls allocate nothing.
struct Arena {
  DevMem mem;
  std::vector<DevMem> overflow;
  size_t off = 0, hwm = 0;
  cudaStream_t st = nullptr;
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

}  // namespace lgs

struct lgs_ctx {
  static constexpr int NSIDE = 12;  // side streams for the independent branches of prove
  int device = 0;
  cudaStream_t st = nullptr;
  cudaStream_t side[NSIDE] = {};
  cudaEvent_t ev_done[NSIDE] = {};
  cudaEvent_t ev_fork = nullptr;
  lgs::DevMem tw;
  lgs::Arena arena;
  lgs::Profiler prof;
  lgs::DevMem err;  // device error word of bounded-wait kernels (0 = ok)
  std::vector<uint8_t> host_stage;  // host copies that must outlive an async upload
  std::vector<uint8_t> host_stage2;
  std::vector<uint8_t> proof_buf;   // the last proof returned by lgs_prove
};

struct lgs_pk {
  lgs::Shape shape;
  lgs::DevMem A;      // 32 x W canonical u64, row-major (the flat A-bar of subset_sum.rs:73-79)
  lgs::DevMem alimb;  // 256 x W bytes: byte l of A[r][k] at row 8r + l
  alignas(64) unsigned char tmap[128];  // TMA descriptor of alimb (CUtensorMap)
  lgs::DevMem a_codes, a_nodes;
  lgs::BasefoldDev a_state;
  lgs::Hash32 com_a;
};

struct lgs_commit_data {
  lgs::Shape shape;
  lgs::DevMem f;      // m x n
  lgs::DevMem cw;     // m x 2n RS codeword F' (its bits are B)
  lgs::DevMem H;      // 32 x 2n digest
  lgs::DevMem nodes;  // column Merkle tree over H
  lgs::Hash32 root;
};
