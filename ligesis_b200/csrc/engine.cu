// Batched and served proving on one GPU.  The reference proves one polynomial at a time on one
// thread (pcs/benches/ligesis.rs:20-60); this engine keeps K lanes - each a full context with its
// own streams and scratch arena, driven by its own host thread - so that commits and proofs of
// many jobs of uneven sizes are in flight on the device together.  A job enters a lane when the
// lane is free and its device-memory estimate fits the engine's HBM budget (FIFO: a job that does
// not fit holds back the ones behind it).  Jobs of one shape share the proving key's device
// buffers read-only.  Every job runs the same commit + prove as lgs_commit / lgs_prove, so its
// proof is byte-identical to the one-at-a-time path.
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "../../include/lgs.h"
#include "prover.cuh"

namespace {
struct EngineJob {
  lgs_job in;
  uint64_t ticket = 0;
  size_t est = 0;
  bool done = false;
  lgs_result res{};
};
}  // namespace

struct lgs_engine {
  int device = 0;
  size_t budget = 0, in_use = 0;
  std::vector<lgs_ctx*> lanes;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<EngineJob*> queue;
  std::unordered_map<uint64_t, EngineJob*> jobs;
  uint64_t next_ticket = 1;
  bool stop = false;
  bool preparing = false;  // lgs_engine_prepare owns the lanes
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

// Device bytes a job holds while it runs: the commitment data (f, codeword, digest, tree) and the
// lane's scratch for the transform and the proof, with margin.
size_t job_estimate(const lgs_pk* pk) {
  const lgs::Shape& s = pk->shape;
  const size_t mn = s.m() * s.n(), ws = s.W() * lgs::NUM_COLS;
  return 48 * mn + 96 * ws + ((size_t)64 << 20);
}

void run_job(lgs_ctx* lane, EngineJob* j) {
  lgs_commit_data cd;
  // The commit is only enqueued: the prove's single synchronisation completes both.
  lgs::commit_dev(lane, j->in.pk, j->in.f, false, &cd, false);
  uint64_t cur[2] = {j->in.cursors[0], j->in.cursors[1]};
  std::vector<uint8_t> proof;
  lgs::prove_dev(lane, j->in.pk, &cd, j->in.z, j->in.zlen, j->in.fields, j->in.nfields, j->in.ints,
                 j->in.nints, cur, &proof);
  lgs::commit_finish(lane, &cd);
  std::memcpy(j->res.root, cd.root.b, 32);
  j->res.proof = (uint8_t*)std::malloc(proof.size() ? proof.size() : 1);
  if (!j->res.proof) throw std::bad_alloc();
  std::memcpy(j->res.proof, proof.data(), proof.size());
  j->res.proof_len = proof.size();
  j->res.cursors[0] = cur[0];
  j->res.cursors[1] = cur[1];
}

void worker_main(lgs_engine* e, size_t lane_idx) {
  cudaSetDevice(e->device);
  lgs_ctx* lane = e->lanes[lane_idx];
  while (true) {
    EngineJob* j = nullptr;
    {
      std::unique_lock<std::mutex> lk(e->mu);
      e->cv_work.wait(lk, [&] {
        return e->stop || (!e->preparing && !e->queue.empty() &&
                           (e->in_use == 0 || e->in_use + e->queue.front()->est <= e->budget));
      });
      if (e->stop) return;
      j = e->queue.front();
      e->queue.pop_front();
      e->in_use += j->est;
      j->res.start_ms = e->now_ms();
    }
    lgs_status st = LGS_OK;
    try {
      run_job(lane, j);
    } catch (...) {
      st = lgs::status_of_current_exception();
    }
    {
      std::lock_guard<std::mutex> lk(e->mu);
      e->in_use -= j->est;
      j->res.status = st;
      j->res.done_ms = e->now_ms();
      j->done = true;
    }
    e->cv_done.notify_all();
    e->cv_work.notify_all();
  }
}

}  // namespace

extern "C" {

lgs_status lgs_engine_create(int device, unsigned lanes, size_t hbm_budget, lgs_engine** out) {
  if (!out || lanes == 0 || lanes > 64)
    return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_create: 1..64 lanes and an output pointer");
  auto* e = new lgs_engine;
  try {
    e->device = device;
    LGS_CUDA(cudaSetDevice(device));
    if (hbm_budget == 0) {
      size_t free_b = 0, total_b = 0;
      LGS_CUDA(cudaMemGetInfo(&free_b, &total_b));
      hbm_budget = free_b / 10 * 9;
    }
    e->budget = hbm_budget;
    for (unsigned i = 0; i < lanes; ++i) {
      auto* c = new lgs_ctx;
      e->lanes.push_back(c);
      lgs::ctx_init(c, device);
      c->copy_pool = false;  // the lanes already copy in parallel
      // larger upload blocks than a lone context: fewer calls per job, the lanes' jobs
      // overlapping each other's uploads instead of their own blocks
      c->upload_block = (size_t)4 << 20;
    }
    for (unsigned i = 0; i < lanes; ++i) e->workers.emplace_back(worker_main, e, (size_t)i);
  } catch (...) {
    lgs_status st = lgs::status_of_current_exception();
    lgs_engine_destroy(e);
    return st;
  }
  *out = e;
  return LGS_OK;
}

void lgs_ctx_destroy(lgs_ctx* ctx);

void lgs_engine_destroy(lgs_engine* e) {
  if (!e) return;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    e->stop = true;
  }
  e->cv_work.notify_all();
  for (auto& w : e->workers)
    if (w.joinable()) w.join();
  for (auto* c : e->lanes) lgs_ctx_destroy(c);
  for (auto& kv : e->jobs) {  // every job not yet collected, queued or finished
    std::free(kv.second->res.proof);
    delete kv.second;
  }
  delete e;
}

lgs_status lgs_engine_submit(lgs_engine* e, const lgs_job* job, uint64_t* ticket) {
  if (!e || !job || !ticket || !job->pk || !job->f || !job->z || !job->fields || !job->ints)
    return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_submit: null argument");
  if (job->len != job->pk->shape.m() * job->pk->shape.n())
    return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_submit: f must hold 2^(log_m+log_n) values");
  if (job->pk->commit_only)
    return lgs::set_error(LGS_ERR_BAD_SHAPE, "lgs_engine_submit: a commit-only key cannot prove");
  auto* j = new EngineJob;
  j->in = *job;
  j->est = job_estimate(job->pk);
  {
    std::lock_guard<std::mutex> lk(e->mu);
    j->ticket = e->next_ticket++;
    j->res.submit_ms = e->now_ms();
    e->jobs[j->ticket] = j;
    e->queue.push_back(j);
  }
  e->cv_work.notify_all();
  *ticket = j->ticket;
  return LGS_OK;
}

lgs_status lgs_engine_wait(lgs_engine* e, uint64_t ticket, double timeout_ms, lgs_result* out) {
  if (!e || !out) return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_wait: null argument");
  std::unique_lock<std::mutex> lk(e->mu);
  auto it = e->jobs.find(ticket);
  if (it == e->jobs.end()) return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_wait: unknown ticket");
  EngineJob* j = it->second;
  auto ready = [&] { return j->done; };
  if (timeout_ms < 0) {
    e->cv_done.wait(lk, ready);
  } else if (!e->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) {
    return lgs::set_error(LGS_ERR_DEVICE_TIMEOUT, "lgs_engine_wait: job not finished in time");
  }
  *out = j->res;  // the proof buffer now belongs to the caller (lgs_engine_free_proof)
  e->jobs.erase(it);
  delete j;
  return LGS_OK;
}

void lgs_engine_free_proof(uint8_t* proof) { std::free(proof); }

lgs_status lgs_engine_prepare(lgs_engine* e, const lgs_pk* const* pks, size_t npk) {
  if (!e || (npk && !pks)) return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_prepare: null argument");
  for (size_t i = 0; i < npk; ++i) {
    if (!pks[i]) return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_prepare: null proving key");
    if (pks[i]->commit_only)
      return lgs::set_error(LGS_ERR_BAD_SHAPE, "lgs_engine_prepare: a commit-only key cannot prove");
  }
  {
    std::lock_guard<std::mutex> lk(e->mu);
    if (!e->queue.empty() || e->in_use != 0 || e->preparing)
      return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_prepare: jobs are queued or running");
    e->preparing = true;
  }
  lgs_status st = LGS_OK;
  try {
    // Synthetic inputs shared by every lane: a zero polynomial of the largest shape, a zero
    // point, distinct oracle ints (so column sampling succeeds) and nonzero fields.
    size_t max_len = 0;
    unsigned max_vars = 0;
    for (size_t i = 0; i < npk; ++i) {
      max_len = std::max(max_len, pks[i]->shape.m() * pks[i]->shape.n());
      max_vars = std::max(max_vars, pks[i]->shape.log_m + pks[i]->shape.log_n);
    }
    const std::vector<lgs::u64> f(max_len, 0), z(2 * (size_t)max_vars, 0);
    size_t nfields = 0;
    for (size_t i = 0; i < npk; ++i) nfields = std::max<size_t>(nfields, lgs::FieldPlan(pks[i]->shape).total);
    std::vector<lgs::u64> fields(2 * nfields);
    for (size_t i = 0; i < fields.size(); ++i) fields[i] = i + 1;
    std::vector<uint64_t> ints(lgs::INTS_PER_PROOF);
    for (size_t i = 0; i < ints.size(); ++i) ints[i] = i;
    std::vector<lgs_status> lane_st(e->lanes.size(), LGS_OK);
    std::vector<std::thread> th;
    for (size_t l = 0; l < e->lanes.size(); ++l)
      th.emplace_back([&, l] {
        try {
          LGS_CUDA(cudaSetDevice(e->device));
          lgs_ctx* lane = e->lanes[l];
          for (int pass = 0; pass < 2; ++pass)  // sizes everything, then captures
            for (size_t i = 0; i < npk; ++i) {
              const lgs::Shape& s = pks[i]->shape;
              lgs_commit_data cd;
              lgs::commit_dev(lane, pks[i], f.data(), false, &cd, false);
              uint64_t cur[2] = {0, 0};
              std::vector<uint8_t> proof;
              lgs::prove_dev(lane, pks[i], &cd, z.data(), s.log_m + s.log_n, fields.data(),
                             nfields, ints.data(), ints.size(), cur, &proof);
              lgs::commit_finish(lane, &cd);
            }
        } catch (...) {
          lane_st[l] = lgs::status_of_current_exception();
        }
      });
    for (auto& t : th) t.join();
    for (lgs_status s : lane_st)
      if (s != LGS_OK) st = s;
  } catch (...) {
    st = lgs::status_of_current_exception();
  }
  {
    std::lock_guard<std::mutex> lk(e->mu);
    e->preparing = false;
  }
  e->cv_work.notify_all();
  return st;
}

lgs_status lgs_engine_tune(lgs_engine* e, const char* name, uint64_t value) {
  if (!e || !name) return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_tune: null argument");
  {
    std::lock_guard<std::mutex> lk(e->mu);
    if (!e->queue.empty() || e->in_use != 0 || e->preparing)
      return lgs::set_error(LGS_ERR_BAD_ARG, "lgs_engine_tune: jobs are queued or running");
    e->preparing = true;  // the workers stay idle while the lanes change
  }
  lgs_status st = LGS_OK;
  for (lgs_ctx* lane : e->lanes) {
    st = lgs_tune(lane, name, value);
    if (st != LGS_OK) break;
  }
  {
    std::lock_guard<std::mutex> lk(e->mu);
    e->preparing = false;
  }
  e->cv_work.notify_all();
  return st;
}

lgs_status lgs_engine_pending(lgs_engine* e, size_t* queued, size_t* running_bytes) {
  if (!e || !queued || !running_bytes) return lgs::set_error(LGS_ERR_BAD_ARG, "null argument");
  std::lock_guard<std::mutex> lk(e->mu);
  *queued = e->queue.size();
  *running_bytes = e->in_use;
  return LGS_OK;
}

}  // extern "C"
