// The extern "C" boundary of liblgs.so (declared in include/lgs.h).  Every entry point catches
// all C++ exceptions and maps them to an lgs_status; the message is kept per host thread.
#include <atomic>
#include <cstring>
#include <new>
#include <string>

#include "../../include/lgs.h"
#include "prover.cuh"

namespace lgs {
int verify_host(unsigned log_m, unsigned log_n, const Hash32& com_a, const Hash32& root,
                const u64* z_in, size_t zlen, const uint8_t* proof, size_t proof_len,
                const u64* fields, size_t nfields, const uint64_t* ints, size_t nints,
                uint64_t cursors[2]);
}  // namespace lgs

using namespace lgs;

namespace {
std::atomic<uint64_t> g_launches{0};
}
thread_local uint64_t t_launches = 0;
void lgs::count_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  ++t_launches;
}
uint64_t lgs::thread_launches() { return t_launches; }
void lgs::adjust_launches(int64_t n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

namespace {
thread_local std::string g_err;

lgs_status fail(lgs_status s, const std::string& m) {
  g_err = m;
  return s;
}

}  // namespace

// Map the exception being handled to a status and record its message (call inside a catch).
lgs_status lgs::status_of_current_exception() {
  try {
    throw;
  } catch (const ShapeError& e) {
    return fail(LGS_ERR_BAD_SHAPE, e.what());
  } catch (const OracleError& e) {
    return fail(LGS_ERR_ORACLE_EXHAUSTED, e.what());
  } catch (const DeviceTimeout& e) {
    return fail(LGS_ERR_DEVICE_TIMEOUT, e.what());
  } catch (const CudaError& e) {
    std::string m = e.what();
    if (m.find("out of memory") != std::string::npos) return fail(LGS_ERR_OOM, m);
    return fail(LGS_ERR_CUDA, m);
  } catch (const std::bad_alloc&) {
    return fail(LGS_ERR_OOM, "host allocation failed");
  } catch (const std::invalid_argument& e) {
    return fail(LGS_ERR_BAD_ARG, e.what());
  } catch (const std::exception& e) {
    return fail(LGS_ERR_INTERNAL, e.what());
  } catch (...) {
    return fail(LGS_ERR_INTERNAL, "unknown exception");
  }
}

namespace {
template <class F>
lgs_status guarded(F&& f) {
  try {
    f();
    return LGS_OK;
  } catch (...) {
    return lgs::status_of_current_exception();
  }
}

}  // namespace

lgs_status lgs::set_error(lgs_status s, const std::string& msg) { return fail(s, msg); }

namespace {
void need(bool c, const char* what) {
  if (!c) throw std::invalid_argument(what);
}

struct CtxDevice {  // make the context's device current for the duration of a call
  int prev = -1;
  explicit CtxDevice(const lgs_ctx* c) {
    cudaGetDevice(&prev);
    if (prev != c->device) LGS_CUDA(cudaSetDevice(c->device));
  }
  ~CtxDevice() {
    int cur;
    if (cudaGetDevice(&cur) == cudaSuccess && prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};
}  // namespace

extern "C" {

const char* lgs_last_error(void) { return g_err.c_str(); }
const char* lgs_version(void) { return "ligesis-b200 0.1 (sm_100a)"; }

lgs_status lgs_ctx_create(int device, unsigned flags, lgs_ctx** out) {
  (void)flags;
  return guarded([&] {
    need(out != nullptr, "lgs_ctx_create: out is null");
    int ndev = 0;
    LGS_CUDA(cudaGetDeviceCount(&ndev));
    need(device >= 0 && device < ndev, "lgs_ctx_create: no such device");
    auto* c = new lgs_ctx;
    try {
      ctx_init(c, device);
    } catch (...) {
      delete c;
      throw;
    }
    *out = c;
  });
}

void lgs_ctx_destroy(lgs_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  if (ctx->hs) cudaStreamSynchronize(ctx->hs);
  // Release the context's own device memory while its stream still exists (the frees are
  // ordered on it), then drain and destroy the streams.
  ctx->prof.flush();
  ctx->arena.overflow.clear();
  ctx->arena.mem.release();
  ctx->tw.release();
  ctx->rs_tw.release();
  ctx->hash_scr.release();
  ctx->err.release();
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  for (int i = 0; i < lgs_ctx::NSIDE; ++i) {
    if (ctx->side[i]) {
      cudaStreamSynchronize(ctx->side[i]);
      cudaStreamDestroy(ctx->side[i]);
    }
    if (ctx->ev_done[i]) cudaEventDestroy(ctx->ev_done[i]);
  }
  for (int i = 0; i < lgs_ctx::RING; ++i)
    if (ctx->ring_ev[i]) cudaEventDestroy(ctx->ring_ev[i]);
  for (int i = 0; i < lgs_ctx::ROW_BLOCKS; ++i)
    if (ctx->ev_rows[i]) cudaEventDestroy(ctx->ev_rows[i]);
  for (int i = 0; i < lgs_ctx::ROW_BLOCKS; ++i)
    if (ctx->ev_rs[i]) cudaEventDestroy(ctx->ev_rs[i]);
  for (int i = 0; i < lgs_ctx::TL_MAX; ++i)
    if (ctx->tl_ev[i]) cudaEventDestroy(ctx->tl_ev[i]);
  for (auto& g : ctx->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  ctx->graphs.clear();
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_fork2) cudaEventDestroy(ctx->ev_fork2);
  if (ctx->ev_cw) cudaEventDestroy(ctx->ev_cw);
  if (ctx->hs) {
    cudaStreamSynchronize(ctx->hs);
    cudaStreamDestroy(ctx->hs);
  }
  for (int i = 0; i < lgs_ctx::NSIDE_HI; ++i)
    if (ctx->side_hi[i]) {
      cudaStreamSynchronize(ctx->side_hi[i]);
      cudaStreamDestroy(ctx->side_hi[i]);
    }
  if (ctx->st) cudaStreamDestroy(ctx->st);
  delete ctx;
}

lgs_status lgs_tensor_peak_i8(lgs_ctx* ctx, unsigned iters, double* tops) {
  return guarded([&] {
    need(ctx && tops && iters >= 1 && iters <= (1u << 20), "lgs_tensor_peak_i8: bad argument");
    CtxDevice dg(ctx);
    *tops = i8_tensor_peak_tops(iters, ctx->err.as<int>(), ctx->st);
    int err = 0;
    LGS_CUDA(cudaMemcpy(&err, ctx->err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
      LGS_CUDA(cudaMemset(ctx->err.p, 0, sizeof(int)));
      throw DeviceTimeout("tensor peak: a bounded device wait gave up");
    }
  });
}

lgs_status lgs_rs_alu_rates(lgs_ctx* ctx, unsigned iters, double* radix8_per_s,
                            double* mul_per_s) {
  return guarded([&] {
    need(ctx && radix8_per_s && mul_per_s && iters >= 1 && iters <= (1u << 24),
         "lgs_rs_alu_rates: bad argument");
    CtxDevice dg(ctx);
    DevMem sink(sizeof(u64), ctx->st);
    *radix8_per_s = rs_alu_rate(0, iters, sink.as<u64>(), ctx->st);
    *mul_per_s = rs_alu_rate(1, iters, sink.as<u64>(), ctx->st);
    LGS_CUDA(cudaStreamSynchronize(ctx->st));
  });
}

lgs_status lgs_ctx_stream(lgs_ctx* ctx, void** stream) {
  return guarded([&] {
    need(ctx && stream, "lgs_ctx_stream: null argument");
    *stream = (void*)ctx->st;
  });
}

lgs_status lgs_setup(lgs_ctx* ctx, unsigned log_m, unsigned log_n, const uint64_t* A,
                     lgs_pk** pk, uint8_t com_a[32]) {
  return guarded([&] {
    need(ctx && A && pk && com_a, "lgs_setup: null argument");
    need(log_m <= 13 && log_n <= 21, "lgs_setup: shape too large");
    CtxDevice dg(ctx);
    auto* k = new lgs_pk;
    try {
      setup_dev(ctx, log_m, log_n, A, k);
    } catch (...) {
      delete k;
      throw;
    }
    std::memcpy(com_a, k->com_a.b, 32);
    *pk = k;
  });
}
lgs_status lgs_setup_commit_only(lgs_ctx* ctx, unsigned log_m, unsigned log_n,
                                 const uint64_t* A, lgs_pk** pk) {
  return guarded([&] {
    need(ctx && A && pk, "lgs_setup_commit_only: null argument");
    need(log_m <= 13 && log_n >= 7 && log_n <= 21,
         "lgs_setup_commit_only: needs log_m <= 13 and 7 <= log_n <= 21");
    CtxDevice dg(ctx);
    auto* k = new lgs_pk;
    try {
      setup_dev(ctx, log_m, log_n, A, k, true);
    } catch (...) {
      delete k;
      throw;
    }
    *pk = k;
  });
}
void lgs_pk_free(lgs_pk* pk) { delete pk; }

static lgs_status commit_impl(lgs_ctx* ctx, const lgs_pk* pk, const uint64_t* f, size_t len,
                              uint8_t root[32], lgs_commit_data** out, bool dev) {
  return guarded([&] {
    need(ctx && pk && f && root && out, "lgs_commit: null argument");
    need(len == pk->shape.m() * pk->shape.n(), "lgs_commit: f must hold 2^(log_m+log_n) values");
    CtxDevice dg(ctx);
    auto* cd = new lgs_commit_data;
    try {
      commit_dev(ctx, pk, f, dev, cd);
    } catch (...) {
      delete cd;
      throw;
    }
    std::memcpy(root, cd->root.b, 32);
    *out = cd;
  });
}
lgs_status lgs_commit(lgs_ctx* ctx, const lgs_pk* pk, const uint64_t* f, size_t len,
                      uint8_t root[32], lgs_commit_data** out) {
  return commit_impl(ctx, pk, f, len, root, out, false);
}
lgs_status lgs_commit_device(lgs_ctx* ctx, const lgs_pk* pk, const uint64_t* f_dev, size_t len,
                             uint8_t root[32], lgs_commit_data** out) {
  return commit_impl(ctx, pk, f_dev, len, root, out, true);
}
lgs_status lgs_commit_async(lgs_ctx* ctx, const lgs_pk* pk, const uint64_t* f, size_t len,
                            int f_on_device, lgs_commit_data** out) {
  return guarded([&] {
    need(ctx && pk && f && out, "lgs_commit_async: null argument");
    need(len == pk->shape.m() * pk->shape.n(),
         "lgs_commit_async: f must hold 2^(log_m+log_n) values");
    need(f_on_device >= 0 && f_on_device <= 2, "lgs_commit_async: f_on_device must be 0, 1 or 2");
    CtxDevice dg(ctx);
    auto* cd = new lgs_commit_data;
    if (f_on_device == 2) cd->f_lent = f;
    try {
      commit_dev(ctx, pk, f, f_on_device != 0, cd, false);
    } catch (...) {
      cudaStreamSynchronize(ctx->st);
      delete cd;
      throw;
    }
    *out = cd;
  });
}
lgs_status lgs_commit_root(lgs_ctx* ctx, lgs_commit_data* cd, uint8_t root[32]) {
  return guarded([&] {
    need(ctx && cd && root, "lgs_commit_root: null argument");
    CtxDevice dg(ctx);
    commit_root(ctx, cd);
    std::memcpy(root, cd->root.b, 32);
  });
}
void lgs_commit_data_free(lgs_commit_data* cd) {
  if (cd && cd->done && !cd->root_ready) cudaEventSynchronize(cd->done);
  delete cd;
}

lgs_status lgs_commit_read(lgs_ctx* ctx, const lgs_commit_data* cd, int which, uint64_t* out,
                           size_t count) {
  return guarded([&] {
    need(ctx && cd && out, "lgs_commit_read: null argument");
    const RecycledBuf& src = which == 0 ? cd->cw : cd->H;
    need(which == 0 || which == 1, "lgs_commit_read: which must be 0 or 1");
    need(count * 8 == src.bytes, "lgs_commit_read: wrong element count");
    CtxDevice dg(ctx);
    if (cd->done) LGS_CUDA(cudaStreamWaitEvent(ctx->st, cd->done, 0));  // H is the hash stream's
    LGS_CUDA(cudaMemcpyAsync(out, src.p, src.bytes, cudaMemcpyDeviceToHost, ctx->st));
    LGS_CUDA(cudaStreamSynchronize(ctx->st));
  });
}

lgs_status lgs_oracle_need(unsigned log_m, unsigned log_n, size_t* fields, size_t* ints) {
  return guarded([&] {
    need(fields && ints, "lgs_oracle_need: null argument");
    Shape s{log_m, log_n};
    if (!s.eval_ok()) throw ShapeError("shape outside the shared-domain window");
    *fields = FieldPlan(s).total;
    *ints = INTS_PER_PROOF;
  });
}

lgs_status lgs_prove(lgs_ctx* ctx, const lgs_pk* pk, const lgs_commit_data* cd,
                     const uint64_t* z, size_t zlen, const uint64_t* fields, size_t nfields,
                     const uint64_t* ints, size_t nints, uint64_t cursors[2],
                     const uint8_t** proof, size_t* proof_len) {
  return guarded([&] {
    need(ctx && pk && cd && z && fields && ints && cursors && proof && proof_len,
         "lgs_prove: null argument");
    if (pk->commit_only) throw ShapeError("lgs_prove: a commit-only key cannot prove");
    CtxDevice dg(ctx);
    uint64_t cur[2] = {cursors[0], cursors[1]};
    std::vector<uint8_t>& buf = ctx->proof_buf;  // reused: written in place by the prove
    prove_dev(ctx, pk, cd, z, zlen, fields, nfields, ints, nints, cur, &buf);
    *proof = buf.data();
    *proof_len = buf.size();
    cursors[0] = cur[0];
    cursors[1] = cur[1];
  });
}

lgs_status lgs_verify(unsigned log_m, unsigned log_n, const uint8_t com_a[32],
                      const uint8_t root[32], const uint64_t* z, size_t zlen,
                      const uint8_t* proof, size_t proof_len, const uint64_t* fields,
                      size_t nfields, const uint64_t* ints, size_t nints, uint64_t cursors[2],
                      int* accept) {
  return guarded([&] {
    need(com_a && root && z && proof && fields && ints && cursors && accept,
         "lgs_verify: null argument");
    Hash32 ca, rt;
    std::memcpy(ca.b, com_a, 32);
    std::memcpy(rt.b, root, 32);
    *accept = verify_host(log_m, log_n, ca, rt, z, zlen, proof, proof_len, fields, nfields, ints,
                          nints, cursors);
  });
}

// ---- standalone Basefold ---------------------------------------------------------------------

lgs_status lgs_basefold_commit(lgs_ctx* ctx, const uint64_t* poly, size_t len, int is_ef,
                               unsigned code_rate, unsigned log_interleave, uint8_t root[32],
                               lgs_basefold** out) {
  return guarded([&] {
    need(ctx && poly && root && out, "lgs_basefold_commit: null argument");
    CtxDevice dg(ctx);
    auto* b = new lgs_basefold;
    try {
      basefold_commit_dev(ctx, poly, len, is_ef != 0, code_rate, log_interleave, b);
    } catch (...) {
      cudaStreamSynchronize(ctx->st);
      delete b;
      throw;
    }
    std::memcpy(root, b->root.b, 32);
    *out = b;
  });
}
void lgs_basefold_free(lgs_basefold* b) { delete b; }

lgs_status lgs_basefold_prove(lgs_ctx* ctx, const lgs_basefold* b, const uint64_t* point,
                              size_t plen, const uint64_t* fields, size_t nfields,
                              const uint64_t* ints, size_t nints, uint64_t cursors[2],
                              const uint8_t** proof, size_t* proof_len) {
  return guarded([&] {
    need(ctx && b && point && fields && ints && cursors && proof && proof_len,
         "lgs_basefold_prove: null argument");
    need(b->device == ctx->device, "lgs_basefold_prove: commitment of another device");
    CtxDevice dg(ctx);
    uint64_t cur[2] = {cursors[0], cursors[1]};
    std::vector<uint8_t>& buf = ctx->proof_buf;
    basefold_prove_dev(ctx, b, point, plen, fields, nfields, ints, nints, cur, &buf);
    *proof = buf.data();
    *proof_len = buf.size();
    cursors[0] = cur[0];
    cursors[1] = cur[1];
  });
}

lgs_status lgs_frac_sum_prove(lgs_ctx* ctx, const uint64_t* p, const uint64_t* q, size_t n,
                              int on_device, const uint64_t* fields, size_t nfields,
                              uint64_t* cursor, const uint8_t** proof, size_t* proof_len,
                              uint64_t* point, uint64_t claim[4]) {
  return guarded([&] {
    need(ctx && q && fields && cursor && proof && proof_len && point && claim,
         "lgs_frac_sum_prove: null argument");
    CtxDevice dg(ctx);
    uint64_t cur = *cursor;
    std::vector<uint8_t>& buf = ctx->proof_buf;
    frac_sum_prove_dev(ctx, p, q, n, on_device != 0, fields, nfields, &cur, &buf, point, claim);
    *proof = buf.data();
    *proof_len = buf.size();
    *cursor = cur;
  });
}

lgs_status lgs_frac_sum_verify(const uint8_t* proof, size_t proof_len, const uint64_t* fields,
                               size_t nfields, uint64_t* cursor, uint64_t* point,
                               size_t point_cap, uint64_t claim[4], int* accept) {
  return guarded([&] {
    need(proof && fields && cursor && point && claim && accept,
         "lgs_frac_sum_verify: null argument");
    *accept = frac_sum_verify_host(proof, proof_len, fields, nfields, cursor, point, point_cap,
                                   claim);
  });
}

lgs_status lgs_lookup_prove(lgs_ctx* ctx, const uint64_t* a, size_t m, const uint64_t* t,
                            const uint64_t* e, size_t n, int on_device, const uint64_t* fields,
                            size_t nfields, uint64_t* cursor, const uint8_t** proof,
                            size_t* proof_len, uint64_t* zq, uint64_t* zt) {
  return guarded([&] {
    need(ctx && a && t && e && fields && cursor && proof && proof_len && zq && zt,
         "lgs_lookup_prove: null argument");
    CtxDevice dg(ctx);
    uint64_t cur = *cursor;
    std::vector<uint8_t>& buf = ctx->proof_buf;
    lookup_prove_dev(ctx, a, m, t, e, n, on_device != 0, fields, nfields, &cur, &buf, zq, zt);
    *proof = buf.data();
    *proof_len = buf.size();
    *cursor = cur;
  });
}

lgs_status lgs_lookup_verify(const uint8_t* proof, size_t proof_len, const uint64_t* fields,
                             size_t nfields, uint64_t* cursor, uint64_t* zq, size_t zq_cap,
                             uint64_t* zt, size_t zt_cap, uint64_t vals[6], int* accept) {
  return guarded([&] {
    need(proof && fields && cursor && zq && zt && vals && accept,
         "lgs_lookup_verify: null argument");
    *accept = lookup_verify_host(proof, proof_len, fields, nfields, cursor, zq, zq_cap, zt,
                                 zt_cap, vals);
  });
}

lgs_status lgs_linear_witness(lgs_ctx* ctx, const int64_t* x, size_t rows, size_t inner,
                              const int64_t* w, size_t cols, int w_transposed,
                              const int64_t* bias, int64_t divisor, int on_device, int64_t* q,
                              int64_t* rem, int64_t* y, uint64_t* y_field) {
  return guarded([&] {
    need(ctx && x && w && q && rem && y, "lgs_linear_witness: null argument");
    CtxDevice dg(ctx);
    linear_witness_dev(ctx, x, rows, inner, w, cols, w_transposed != 0, bias, divisor,
                       on_device != 0, q, rem, y, y_field);
  });
}

lgs_status lgs_layer_norm_witness(lgs_ctx* ctx, const int64_t* x, size_t rows, size_t d,
                                  const int64_t* gain, const int64_t* bias, int on_device,
                                  int64_t* sum_x, int64_t* sum_x2, int64_t* var_sum,
                                  int64_t* stdv, int64_t* dividend, int64_t* quotient,
                                  int64_t* output) {
  return guarded([&] {
    need(ctx && x && gain && bias && sum_x && sum_x2 && var_sum && stdv && dividend && quotient &&
             output,
         "lgs_layer_norm_witness: null argument");
    CtxDevice dg(ctx);
    int64_t* const rows_out[4] = {sum_x, sum_x2, var_sum, stdv};
    int64_t* const ent_out[3] = {dividend, quotient, output};
    layer_norm_witness_dev(ctx, x, rows, d, gain, bias, on_device != 0, rows_out, ent_out);
  });
}

lgs_status lgs_softmax_witness(lgs_ctx* ctx, const int64_t* scores, unsigned heads, unsigned n,
                               const int64_t* exp_lut, size_t lut_len, int64_t offset,
                               int64_t scale, int on_device, int64_t* x_max, int64_t* exp,
                               int64_t* sum_exp, int64_t* prob) {
  return guarded([&] {
    need(ctx && scores && exp_lut && x_max && exp && sum_exp && prob,
         "lgs_softmax_witness: null argument");
    CtxDevice dg(ctx);
    softmax_witness_dev(ctx, scores, heads, n, exp_lut, lut_len, offset, scale, on_device != 0,
                        x_max, exp, sum_exp, prob);
  });
}

lgs_status lgs_lut_gather(lgs_ctx* ctx, const int64_t* v, size_t count, const int64_t* lut,
                          size_t lut_len, int64_t offset, int on_device, int64_t* out) {
  return guarded([&] {
    need(ctx && v && lut && out, "lgs_lut_gather: null argument");
    CtxDevice dg(ctx);
    lut_gather_dev(ctx, v, count, lut, lut_len, offset, on_device != 0, out);
  });
}

lgs_status lgs_basefold_verify(const uint8_t root[32], const uint64_t* point, size_t plen,
                               const uint8_t* proof, size_t proof_len, const uint64_t* fields,
                               size_t nfields, const uint64_t* ints, size_t nints,
                               uint64_t cursors[2], int* accept) {
  return guarded([&] {
    need(root && point && proof && fields && ints && cursors && accept,
         "lgs_basefold_verify: null argument");
    Hash32 rt;
    std::memcpy(rt.b, root, 32);
    *accept = basefold_verify_host(rt, point, plen, proof, proof_len, fields, nfields, ints, nints,
                                   cursors);
  });
}

// ---- measurement ----------------------------------------------------------------------------

namespace {
// Waits for the context's streams and folds the stage events they recorded into the totals
// (an asynchronous commit's stages are otherwise folded in only by a later call).
void profile_settle(lgs_ctx* ctx) {
  CtxDevice dg(ctx);
  LGS_CUDA(cudaStreamSynchronize(ctx->st));
  LGS_CUDA(cudaStreamSynchronize(ctx->hs));
  ctx->prof.flush();
}
}  // namespace

lgs_status lgs_profile(lgs_ctx* ctx, int enable) {
  return guarded([&] {
    need(ctx != nullptr, "lgs_profile: null context");
    CtxDevice dg(ctx);
    LGS_CUDA(cudaStreamSynchronize(ctx->st));
    ctx->prof.flush();
    ctx->prof.totals.clear();
    ctx->prof.on = enable != 0;
    ctx->prof_level = enable;
  });
}

lgs_status lgs_profile_names(lgs_ctx* ctx, char* buf, size_t cap, size_t* needed) {
  return guarded([&] {
    need(ctx && needed, "lgs_profile_names: null argument");
    profile_settle(ctx);
    std::string all;
    for (auto& t : ctx->prof.totals) all += t.first + "\n";
    *needed = all.size() + 1;
    if (buf && cap) {
      const size_t nb = std::min(cap - 1, all.size());
      std::memcpy(buf, all.data(), nb);
      buf[nb] = 0;
    }
  });
}

lgs_status lgs_tune(lgs_ctx* ctx, const char* name, uint64_t value) {
  return guarded([&] {
    need(ctx && name, "lgs_tune: null argument");
    const std::string n(name);
    if (n == "hash_ctas") {
      need(value <= 4096, "lgs_tune: hash_ctas above 4096");
      ctx->hash_ctas = (unsigned)value;
    } else if (n == "hash_groups") {
      need(value <= lgs_ctx::ROW_BLOCKS, "lgs_tune: hash_groups above the upload's row blocks");
      ctx->hash_groups = (unsigned)value;
    } else if (n == "witness_path") {
      need(value <= 1, "lgs_tune: witness_path is 0 (tensor cores) or 1 (CUDA cores)");
      ctx->witness_path = (unsigned)value;
    } else if (n == "upload_block_bytes") {
      need(value <= ((uint64_t)1 << 40), "lgs_tune: upload_block_bytes above 2^40");
      ctx->upload_block = (size_t)value;
    } else if (n == "upload_tail_rows") {
      need(value <= 65536, "lgs_tune: upload_tail_rows above 65536");
      ctx->upload_tail = (size_t)value;
    } else if (n == "witness_ctas") {
      need(value <= 65536, "lgs_tune: witness_ctas above 65536");
      ctx->witness_ctas = (unsigned)value;
    } else if (n == "sumcheck_blocks") {
      need(value <= SC_MAX_BLOCKS, "lgs_tune: sumcheck_blocks above the partial-sum slots");
      ctx->sumcheck_blocks = (unsigned)value;
      // captured prove graphs hold the old launch shapes: drop them (recaptured on next use)
      CtxDevice dg(ctx);
      LGS_CUDA(cudaStreamSynchronize(ctx->st));
      for (auto& g : ctx->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
      ctx->graphs.clear();
    } else {
      throw std::invalid_argument("lgs_tune: unknown parameter " + n);
    }
  });
}

lgs_status lgs_tune_get(lgs_ctx* ctx, const char* name, uint64_t* value) {
  return guarded([&] {
    need(ctx && name && value, "lgs_tune_get: null argument");
    const std::string n(name);
    if (n == "hash_ctas") *value = ctx->hash_ctas;
    else if (n == "sumcheck_blocks") *value = ctx->sumcheck_blocks;
    else if (n == "hash_groups") *value = ctx->hash_groups;
    else if (n == "witness_path") *value = ctx->witness_path;
    else if (n == "witness_ctas") *value = ctx->witness_ctas;
    else if (n == "upload_block_bytes") *value = ctx->upload_block;
    else if (n == "upload_tail_rows") *value = ctx->upload_tail;
    else throw std::invalid_argument("lgs_tune_get: unknown parameter " + n);
  });
}

lgs_status lgs_set_wait_budget(lgs_ctx* ctx, uint64_t cycles) {
  return guarded([&] {
    need(ctx != nullptr, "lgs_set_wait_budget: null context");
    ctx->wait_cycles = cycles;
  });
}

lgs_status lgs_profile_get(lgs_ctx* ctx, const char* stage, double* total_ms, uint64_t* count) {
  return guarded([&] {
    need(ctx && stage && total_ms && count, "lgs_profile_get: null argument");
    profile_settle(ctx);
    *total_ms = 0;
    *count = 0;
    for (auto& t : ctx->prof.totals)
      if (t.first == stage) {
        *total_ms = t.second.first;
        *count = t.second.second;
      }
  });
}

uint64_t lgs_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

// ---- individual operations ----------------------------------------------------------------

lgs_status lgs_dft(lgs_ctx* ctx, const uint64_t* in, size_t n_in, size_t batch,
                   unsigned log_size, uint64_t* out) {
  return guarded([&] {
    need(ctx && in && out, "lgs_dft: null argument");
    need(log_size >= 1 && log_size <= TW_LOG, "lgs_dft: size out of range");
    const size_t N = (size_t)1 << log_size;
    need(n_in >= 1 && n_in <= N && batch >= 1, "lgs_dft: bad lengths");
    CtxDevice dg(ctx);
    ctx->arena.begin();
    u64* d_in = ctx->arena.get<u64>(batch * n_in);
    u64* d_out = ctx->arena.get<u64>(batch * N);
    u64* scr = log_size > 12 ? ctx->arena.get<u64>(batch * N) : nullptr;
    std::vector<u64> canon(in, in + batch * n_in);
    for (auto& x : canon) x = gl_canon(x);
    LGS_CUDA(cudaMemcpyAsync(d_in, canon.data(), canon.size() * 8, cudaMemcpyHostToDevice, ctx->st));
    if (rs_dft_supported(log_size, n_in))
      rs_dft_rows(d_in, n_in, n_in, d_out, N, log_size, batch, scr, ctx->rs_tw.as<u64>(), ctx->st);
    else
      ntt_batch(d_in, n_in, n_in, d_out, N, log_size, batch, scr, ctx->tw.as<u64>(), ctx->st);
    LGS_CUDA(cudaMemcpyAsync(out, d_out, batch * N * 8, cudaMemcpyDeviceToHost, ctx->st));
    LGS_CUDA(cudaStreamSynchronize(ctx->st));
  });
}

lgs_status lgs_subset_sum_hash(lgs_ctx* ctx, const uint64_t* A, size_t m, const uint64_t* cw,
                               size_t cols, uint64_t* H) {
  return guarded([&] {
    need(ctx && A && cw && H, "lgs_subset_sum_hash: null argument");
    need(m >= 1 && m <= 8192 && cols >= 1, "lgs_subset_sum_hash: 1 <= m <= 8192, cols >= 1");
    CtxDevice dg(ctx);
    const size_t W = 64 * m, cp = (cols + 255) / 256 * 256;  // kernel tile: 256 columns
    ctx->arena.begin();
    u64* dA = ctx->arena.get<u64>(DIGEST_ROWS * W);
    uint8_t* dL = ctx->arena.get<uint8_t>(DIGEST_ROWS * W * 8);
    u64* dC = ctx->arena.get<u64>(m * cp);
    u64* dH = ctx->arena.get<u64>(DIGEST_ROWS * cp);
    u32* dN = ctx->arena.get<u32>(cp * 8);
    std::vector<u64> a(A, A + DIGEST_ROWS * W), c(cw, cw + m * cols);
    for (auto& x : a) x = gl_canon(x);
    for (auto& x : c) x = gl_canon(x);
    LGS_CUDA(cudaMemcpyAsync(dA, a.data(), a.size() * 8, cudaMemcpyHostToDevice, ctx->st));
    LGS_CUDA(cudaMemsetAsync(dC, 0, m * cp * 8, ctx->st));
    LGS_CUDA(cudaMemcpy2DAsync(dC, cp * 8, c.data(), cols * 8, cols * 8, m,
                               cudaMemcpyHostToDevice, ctx->st));
    alimb_from_a(dA, dL, W, ctx->st);
    alignas(64) unsigned char tmap[128];
    make_alimb_tmap(dL, W, tmap);
    const unsigned splits = subset_sum_hash_splits(cp, (unsigned)m, ctx->hash_ctas);
    u64* slices = splits > 1 ? ctx->arena.get<u64>((size_t)splits * DIGEST_ROWS * cp) : nullptr;
    subset_sum_hash_tc(tmap, dC, dH, dN, (unsigned)m, cp, ctx->err.as<int>(), ctx->st,
                       ctx->wait_cycles, ctx->hash_ctas, 0, 0, 2, slices);
    LGS_CUDA(cudaMemcpy2DAsync(H, cols * 8, dH, cp * 8, cols * 8, DIGEST_ROWS,
                               cudaMemcpyDeviceToHost, ctx->st));
    int err = 0;
    LGS_CUDA(cudaMemcpyAsync(&err, ctx->err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    LGS_CUDA(cudaStreamSynchronize(ctx->st));
    if (err) {
      LGS_CUDA(cudaMemsetAsync(ctx->err.p, 0, sizeof(int), ctx->st));
      throw DeviceTimeout("subset-sum hash: a bounded device wait gave up");
    }
  });
}

lgs_status lgs_merkle_root(lgs_ctx* ctx, const uint64_t* leaves, size_t nleaves, unsigned words,
                           uint8_t root[32]) {
  return guarded([&] {
    need(ctx && leaves && root, "lgs_merkle_root: null argument");
    need(nleaves >= 1 && (nleaves & (nleaves - 1)) == 0, "lgs_merkle_root: nleaves must be a power of two");
    need(words >= 1 && words * 8 <= 1024, "lgs_merkle_root: leaf must be 8..1024 bytes");
    CtxDevice dg(ctx);
    ctx->arena.begin();
    u64* d = ctx->arena.get<u64>(nleaves * words);
    u32* nodes = ctx->arena.get<u32>((2 * nleaves - 1) * 8);
    LGS_CUDA(cudaMemcpyAsync(d, leaves, nleaves * words * 8, cudaMemcpyHostToDevice, ctx->st));
    merkle_leaves_contig(d, words, nleaves, nodes, ctx->st);
    merkle_build_from_leaves(nodes, nleaves, ctx->st);
    LGS_CUDA(cudaMemcpyAsync(root, nodes + (2 * nleaves - 2) * 8, 32, cudaMemcpyDeviceToHost, ctx->st));
    LGS_CUDA(cudaStreamSynchronize(ctx->st));
  });
}

lgs_status lgs_sumcheck_prove(lgs_ctx* ctx, const uint64_t* polys, unsigned d, unsigned k,
                              const uint64_t* challenges, uint64_t* rounds_out,
                              uint64_t* finals_out) {
  return guarded([&] {
    need(ctx && polys && challenges && rounds_out && finals_out, "lgs_sumcheck_prove: null argument");
    need(d >= 1 && d <= 3 && k >= 1 && k <= 30, "lgs_sumcheck_prove: 1..3 factors, 1..30 variables");
    CtxDevice dg(ctx);
    const size_t len = (size_t)1 << k;
    ctx->arena.begin();
    ef2* p[3];
    for (unsigned j = 0; j < d; ++j) p[j] = ctx->arena.get<ef2>(len);
    ef2* ch = ctx->arena.get<ef2>(k);
    ef2* ro = ctx->arena.get<ef2>((size_t)k * (d + 1));
    ef2* fo = ctx->arena.get<ef2>(d);
    ef2* part = ctx->arena.get<ef2>(sumcheck_partials_elems(k, d));
    std::vector<u64> hp(polys, polys + 2 * len * d), hc(challenges, challenges + 2 * k);
    for (auto& x : hp) x = gl_canon(x);
    for (auto& x : hc) x = gl_canon(x);
    for (unsigned j = 0; j < d; ++j)
      LGS_CUDA(cudaMemcpyAsync(p[j], hp.data() + 2 * len * j, len * 16, cudaMemcpyHostToDevice, ctx->st));
    LGS_CUDA(cudaMemcpyAsync(ch, hc.data(), k * 16, cudaMemcpyHostToDevice, ctx->st));
    sumcheck_prove_dev(p, d, k, ch, ro, fo, part, ctx->st);
    LGS_CUDA(cudaMemcpyAsync(rounds_out, ro, (size_t)k * (d + 1) * 16, cudaMemcpyDeviceToHost, ctx->st));
    LGS_CUDA(cudaMemcpyAsync(finals_out, fo, d * 16, cudaMemcpyDeviceToHost, ctx->st));
    LGS_CUDA(cudaStreamSynchronize(ctx->st));
  });
}

// ---- device-resident forms (inputs already in HBM; enqueued on the context's stream) ----------
lgs_status lgs_sumcheck_prove_dev(lgs_ctx* ctx, uint64_t* polys_dev, unsigned d, unsigned k,
                                  const uint64_t* challenges_dev, uint64_t* rounds_out_dev,
                                  uint64_t* finals_out_dev) {
  return guarded([&] {
    need(ctx && polys_dev && challenges_dev && rounds_out_dev && finals_out_dev,
         "lgs_sumcheck_prove_dev: null argument");
    need(d >= 1 && d <= 3 && k >= 1 && k <= 30, "lgs_sumcheck_prove_dev: 1..3 factors, 1..30 variables");
    CtxDevice dg(ctx);
    const size_t len = (size_t)1 << k;
    ctx->arena.begin();
    ef2* part = ctx->arena.get<ef2>(sumcheck_partials_elems(k, d));
    ef2* p[3];
    for (unsigned j = 0; j < d; ++j) p[j] = (ef2*)polys_dev + j * len;
    sumcheck_prove_dev(p, d, k, (const ef2*)challenges_dev, (ef2*)rounds_out_dev,
                       (ef2*)finals_out_dev, part, ctx->st);
  });
}

lgs_status lgs_new_eq_dev(lgs_ctx* ctx, const uint64_t* point_dev, unsigned k, uint64_t* out_dev) {
  return guarded([&] {
    need(ctx && point_dev && out_dev, "lgs_new_eq_dev: null argument");
    need(k >= 1 && k <= 30, "lgs_new_eq_dev: 1..30 variables");
    CtxDevice dg(ctx);
    new_eq_dev((const ef2*)point_dev, k, (ef2*)out_dev, ctx->st);
  });
}

lgs_status lgs_mle_fold_dev(lgs_ctx* ctx, const uint64_t* evals_dev, unsigned k,
                            const uint64_t* point_dev, unsigned np, uint64_t* out_dev) {
  return guarded([&] {
    need(ctx && evals_dev && point_dev && out_dev, "lgs_mle_fold_dev: null argument");
    need(k >= 1 && k <= 30, "lgs_mle_fold_dev: 1..30 variables");
    CtxDevice dg(ctx);
    mle_fold_dev((const ef2*)evals_dev, k, (const ef2*)point_dev, np, (ef2*)out_dev, ctx->st);
  });
}

lgs_status lgs_mle_eval_dev(lgs_ctx* ctx, const uint64_t* evals_dev, unsigned k,
                            const uint64_t* point_dev, uint64_t* out_dev) {
  return guarded([&] {
    need(ctx && evals_dev && point_dev && out_dev, "lgs_mle_eval_dev: null argument");
    need(k >= 1 && k <= 30, "lgs_mle_eval_dev: 1..30 variables");
    CtxDevice dg(ctx);
    ctx->arena.begin();
    ef2* part = ctx->arena.get<ef2>(eqdot_partials_elems(k));
    eq_dot_dev(evals_dev, 0, (const ef2*)point_dev, k, (ef2*)out_dev, part, ctx->st);
  });
}

lgs_status lgs_mle_eval(lgs_ctx* ctx, const uint64_t* evals, unsigned k, const uint64_t* point,
                        uint64_t out[2]) {
  return guarded([&] {
    need(ctx && evals && point && out, "lgs_mle_eval: null argument");
    need(k >= 1 && k <= 30, "lgs_mle_eval: 1..30 variables");
    CtxDevice dg(ctx);
    const size_t len = (size_t)1 << k;
    ctx->arena.begin();
    ef2* v = ctx->arena.get<ef2>(len);
    ef2* pt = ctx->arena.get<ef2>(k);
    ef2* o = ctx->arena.get<ef2>(1);
    ef2* part = ctx->arena.get<ef2>(eqdot_partials_elems(k));
    std::vector<u64> hv(evals, evals + 2 * len), hp(point, point + 2 * k);
    for (auto& x : hv) x = gl_canon(x);
    for (auto& x : hp) x = gl_canon(x);
    LGS_CUDA(cudaMemcpyAsync(v, hv.data(), len * 16, cudaMemcpyHostToDevice, ctx->st));
    LGS_CUDA(cudaMemcpyAsync(pt, hp.data(), k * 16, cudaMemcpyHostToDevice, ctx->st));
    eq_dot_dev(v, 0, pt, k, o, part, ctx->st);
    LGS_CUDA(cudaMemcpyAsync(out, o, 16, cudaMemcpyDeviceToHost, ctx->st));
    LGS_CUDA(cudaStreamSynchronize(ctx->st));
  });
}

lgs_status lgs_new_eq(lgs_ctx* ctx, const uint64_t* point, unsigned k, uint64_t* out) {
  return guarded([&] {
    need(ctx && point && out, "lgs_new_eq: null argument");
    need(k >= 1 && k <= 30, "lgs_new_eq: 1..30 variables");
    CtxDevice dg(ctx);
    const size_t len = (size_t)1 << k;
    ctx->arena.begin();
    ef2* pt = ctx->arena.get<ef2>(k);
    ef2* o = ctx->arena.get<ef2>(len);
    std::vector<u64> hp(point, point + 2 * k);
    for (auto& x : hp) x = gl_canon(x);
    LGS_CUDA(cudaMemcpyAsync(pt, hp.data(), k * 16, cudaMemcpyHostToDevice, ctx->st));
    new_eq_dev(pt, k, o, ctx->st);
    LGS_CUDA(cudaMemcpyAsync(out, o, len * 16, cudaMemcpyDeviceToHost, ctx->st));
    LGS_CUDA(cudaStreamSynchronize(ctx->st));
  });
}

}  // extern "C"
