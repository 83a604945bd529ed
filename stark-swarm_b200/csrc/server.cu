// server.cu — continuous-batching proof server (many proofs in flight on one GPU).
//
// The reference proves one shard per worker process and scales across
// processes (swarm-worker, swarm-ctrl). On one B200 a single small proof
// (n0 = 2^12..2^17) occupies a few SMs and spends most of its latency in
// Fiat-Shamir round trips, so throughput comes from keeping many proofs in
// flight: N worker threads, each with its own CUDA stream and context
// (sharing the parent's twiddle tables), take jobs from a FIFO queue as soon
// as they finish the previous one. Admission is by HBM footprint: a job starts
// only while the footprints of the running jobs plus its own stay within the
// budget (a job larger than the whole budget runs alone). Results are byte
// for byte those of the single-proof entry points.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "context.hpp"
#include "ed25519.hpp"
#include "ed25519_prover.hpp"
#include "p256.hpp"
#include "p256_prover.hpp"
#include "prover.hpp"
#include "rsa2048.hpp"
#include "sha256_air.cuh"
#include "sha512_air.cuh"
#include "verifier.hpp"

namespace {

using Clock = std::chrono::steady_clock;

struct Entry {
  int32_t kind = 0;
  int32_t phi_mode = 0;
  uint64_t blowup = 32;
  uint32_t flags = 0;   // SG_JOB_FAULT_* (tests)
  int attempts = 0;     // runs started
  bool cancel = false;  // cancelled while running: the result is discarded
  std::vector<uint8_t> input;
  uint8_t pi[32];
  uint64_t footprint = 0;
  bool done = false;
  int status = SG_OK;
  std::string err;
  std::vector<uint8_t> proof;
  uint8_t digest[64] = {0};
  Clock::time_point t_submit, t_start, t_end;
};

uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

uint64_t job_blowup(const sg_job& j) { return j.blowup && j.kind != SG_JOB_HASH_ROLLUP ? j.blowup : 32; }

// Device bytes a job holds at its peak (LDE + trace + quotient + STIR buffers), estimated.
uint64_t footprint_bytes(const sg_job& j) {
  const uint64_t bu = job_blowup(j);
  if (j.kind == SG_JOB_SHA256) {
    const uint64_t blocks = (j.input_len + 9 + 63) / 64;
    const uint64_t nt = next_pow2(128 * blocks), n0 = nt * bu;
    return 8 * ((uint64_t)sg::sha::WIDTH * (n0 + 2 * nt) + 16 * n0);
  }
  if (j.kind == SG_JOB_SHA512) {
    const uint64_t blocks = (j.input_len + 17 + 127) / 128;
    const uint64_t nt = next_pow2(128 * blocks), n0 = nt * bu;
    return 8 * ((uint64_t)sg::sha512::WIDTH * (n0 + 2 * nt) + 16 * n0);
  }
  if (j.kind == SG_JOB_P256_ECDSA) {
    // trace, coefficients and LDE at 151,334 columns (the LDE is evaluated
    // coset by coset, without a scratch copy)
    return 8ull * sg::p256::layout().width * (2 * sg::p256::K_ECDSA + sg::p256::K_ECDSA * bu) + (64ull << 20);
  }
  if (j.kind == SG_JOB_RSA2048) {
    const uint64_t recs = j.input_len / 768, w = recs * sg::rsa::WIDTH, n0 = sg::rsa::N_TRACE * bu;
    return 8 * (w * (sg::rsa::N_TRACE + n0) + (recs + 16) * n0);
  }
  if (j.kind == SG_JOB_ED25519) {
    // trace and the materialised LDE at the layout's width, quotient and STIR buffers
    const sg::ed25519::Layout L = sg::ed25519::make_layout(j.input_len - 32, sg::ed25519::K_FULL);
    const uint64_t n0 = (uint64_t)L.height * bu;
    return 8 * ((uint64_t)L.width * (L.height + n0) + 16 * n0) + (64ull << 20);
  }
  const uint64_t nt = next_pow2(j.input_len < 8 ? 8 : j.input_len), n0 = nt * 32;
  return 8 * (4 * n0 + 8 * nt + 16 * n0);
}

// pub || sig || msg: the native check first (prove_zsk_ksk_binding_v2 refuses an
// invalid signature before proving, swarm-dns/src/prover.rs:870-876)
void check_ed25519_job(const std::vector<uint8_t>& in) {
  if (!sg::ed25519::verify(in.data(), in.data() + 32, in.data() + 96, in.size() - 96))
    throw sg::SgError{SG_EVERIFY, "ed25519 job: the signature does not verify"};
}

// n || s || em per record (256 bytes each) -> the three contiguous arrays prove_rsa2048 takes
std::vector<uint8_t> prove_rsa_job(sg_ctx* c, const std::vector<uint8_t>& in, const uint8_t pi[32], uint64_t blowup,
                                   bool self_verify) {
  const uint64_t recs = in.size() / 768;
  std::vector<uint8_t> n(256 * recs), s(256 * recs), em(256 * recs);
  for (uint64_t r = 0; r < recs; ++r) {
    memcpy(&n[256 * r], &in[768 * r], 256);
    memcpy(&s[256 * r], &in[768 * r + 256], 256);
    memcpy(&em[256 * r], &in[768 * r + 512], 256);
  }
  return sg::prove_rsa2048(c, n.data(), s.data(), em.data(), recs, pi, self_verify, blowup);
}

}  // namespace

struct sg_server {
  sg_ctx* parent = nullptr;
  int max_retries = 0;
  int group_max = 1;  // SG_OPT_STIR_GROUP of the parent context
  uint64_t budget = 0;
  uint64_t in_flight = 0;
  int running = 0;
  bool stop = false;
  uint64_t next_ticket = 1;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> queue;
  std::map<uint64_t, Entry> entries;
  std::vector<sg_ctx*> wctx;
  std::vector<std::thread> threads;

  void worker(sg_ctx* c) {
    cudaSetDevice(c->device);
    for (;;) {
      std::vector<uint64_t> tickets;
      std::vector<Entry*> es;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] {
          if (stop) return true;
          if (queue.empty()) return false;
          const Entry& f = entries.at(queue.front());
          return running == 0 || in_flight + f.footprint <= budget;
        });
        if (stop) return;
        auto take = [&](uint64_t t) {
          Entry* x = &entries.at(t);
          tickets.push_back(t);
          es.push_back(x);
          in_flight += x->footprint;
          ++x->attempts;
          if (x->attempts == 1) x->t_start = Clock::now();
        };
        take(queue.front());
        queue.pop_front();
        // lockstep STIR: further queued jobs with the same n0, as far as the budget allows
        const uint64_t n0 = job_n0(*es[0]);
        if (group_max > 1 && n0) {
          for (auto q = queue.begin(); q != queue.end() && (int)es.size() < group_max;) {
            const Entry& f = entries.at(*q);
            if (job_n0(f) == n0 && in_flight + f.footprint <= budget) {
              take(*q);
              q = queue.erase(q);
            } else {
              ++q;
            }
          }
        }
        ++running;
      }
      if (es.size() == 1)
        run(c, es[0]);
      else
        run_group(c, es);
      {
        std::lock_guard<std::mutex> lk(mu);
        --running;
        for (size_t i = 0; i < es.size(); ++i) {
          Entry* e = es[i];
          in_flight -= e->footprint;
          const bool transient = e->status == SG_ENOMEM || e->status == SG_ECUDA;
          if (e->cancel) {
            e->status = SG_ECANCELED;
            e->proof.clear();
          } else if (transient && e->attempts <= max_retries) {
            // reopened: back to the head of the queue for another attempt
            queue.push_front(tickets[i]);
            continue;
          }
          e->t_end = Clock::now();
          e->done = true;
        }
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }

  // The proof domain of a job that can join a lockstep STIR group (0: it cannot).
  static uint64_t job_n0(const Entry& e) {
    if (e.kind == SG_JOB_SHA256)
      return next_pow2(128 * ((e.input.size() + 9 + 63) / 64)) * e.blowup;
    if (e.kind == SG_JOB_SHA512)
      return next_pow2(128 * ((e.input.size() + 17 + 127) / 128)) * e.blowup;
    if (e.kind == SG_JOB_P256_ECDSA) return sg::p256::K_ECDSA * e.blowup;
    if (e.kind == SG_JOB_RSA2048) return sg::rsa::N_TRACE * e.blowup;
    if (e.kind == SG_JOB_ED25519)
      return (uint64_t)sg::ed25519::make_layout(e.input.size() - 32, sg::ed25519::K_FULL).height * e.blowup;
    return 0;
  }

  // A job's c_eval (everything before its STIR phase).
  static sg::CEval ceval(sg_ctx* c, Entry* e) {
    const uint8_t* in = e->input.data();
    if (e->kind == SG_JOB_SHA256)
      return sg::hash_message_ceval(c, sg::sha256_hash_air(), in, e->input.size(), e->pi, e->phi_mode, e->digest,
                                    e->blowup);
    if (e->kind == SG_JOB_SHA512)
      return sg::hash_message_ceval(c, sg::sha512_hash_air(), in, e->input.size(), e->pi, e->phi_mode, e->digest,
                                    e->blowup);
    if (e->kind == SG_JOB_P256_ECDSA)
      return sg::p256_ecdsa_ceval(c, in, in + 32, in + 64, in + 96, in + 128, e->pi, e->blowup);
    if (e->kind == SG_JOB_ED25519) {
      check_ed25519_job(e->input);
      return sg::ed25519_ceval(c, in, in + 32, in + 96, e->input.size() - 96, e->pi, sg::ed25519::K_FULL,
                               e->blowup);
    }
    const uint64_t recs = e->input.size() / 768;
    std::vector<uint8_t> n(256 * recs), s(256 * recs), em(256 * recs);
    for (uint64_t r = 0; r < recs; ++r) {
      memcpy(&n[256 * r], &in[768 * r], 256);
      memcpy(&s[256 * r], &in[768 * r + 256], 256);
      memcpy(&em[256 * r], &in[768 * r + 512], 256);
    }
    return sg::rsa2048_ceval(c, n.data(), s.data(), em.data(), recs, e->pi, e->blowup);
  }

  // Jobs with one n0: each c_eval on its own, then one lockstep STIR phase for all
  // of them, then each proof's self-verification. A job that fails before the STIR
  // phase leaves the group; a failure of the group's STIR phase fails its jobs.
  static void run_group(sg_ctx* c, const std::vector<Entry*>& es) {
    std::vector<Entry*> ok;
    std::vector<sg::CEval> ce;
    for (Entry* e : es) {
      e->proof.clear();
      e->err.clear();
      try {
        if ((e->flags & SG_JOB_FAULT_ALLOC) && e->attempts == 1)
          throw sg::SgError{SG_ENOMEM, "injected fault: device allocation failed"};
        ce.push_back(ceval(c, e));
        ok.push_back(e);
      } catch (const sg::SgError& x) {
        e->status = x.code;
        e->err = x.msg;
      } catch (const std::exception& x) {
        e->status = SG_EINVAL;
        e->err = x.what();
      }
    }
    if (ok.empty()) return;
    try {
      const uint64_t n0 = ce[0].n0;
      sg::DBuf f0(n0 * ok.size(), c->stream);
      std::vector<sg_fri_params> ps;
      for (size_t g = 0; g < ok.size(); ++g) {
        sg::require(ce[g].n0 == n0, "stir group: mixed domains");
        sg::cuda_check(cudaMemcpyAsync(f0.p + g * n0, ce[g].d_c.p, n0 * 8, cudaMemcpyDeviceToDevice, c->stream),
                       "copy");
        ps.push_back(ce[g].params);
      }
      ce.clear();
      std::vector<std::vector<uint8_t>> proofs = sg::stir_prove_group(c, f0.p, n0, n0, ps);
      for (size_t g = 0; g < ok.size(); ++g) {
        Entry* e = ok[g];
        e->proof = std::move(proofs[g]);
        if (e->flags & SG_JOB_FAULT_VERIFY) e->proof[e->proof.size() / 2] ^= 0x40;
        try {
          const sg::StirProof pr = sg::decode_proof(e->proof.data(), e->proof.size());
          e->status = sg::stir_verify(pr, ps[g]) ? SG_OK : SG_EVERIFY;
        } catch (const std::exception&) {
          e->status = SG_EVERIFY;
        }
        if (e->status != SG_OK) e->err = "self-verification of the produced proof failed";
      }
    } catch (const sg::SgError& x) {
      for (Entry* e : ok) {
        e->status = x.code;
        e->err = x.msg;
      }
    } catch (const std::exception& x) {
      for (Entry* e : ok) {
        e->status = SG_EINVAL;
        e->err = x.what();
      }
    }
  }

  static void run(sg_ctx* c, Entry* e) {
    e->proof.clear();
    e->err.clear();
    try {
      if ((e->flags & SG_JOB_FAULT_ALLOC) && e->attempts == 1)
        throw sg::SgError{SG_ENOMEM, "injected fault: device allocation failed"};
      prove(c, e, !(e->flags & SG_JOB_FAULT_VERIFY));
      if (e->flags & SG_JOB_FAULT_VERIFY) {
        // a corrupted proof goes through the same self-verification as every proof
        require_nonempty(e->proof);
        e->proof[e->proof.size() / 2] ^= 0x40;
        const sg::StirProof pr = sg::decode_proof(e->proof.data(), e->proof.size());
        sg_fri_params p;
        sg_build_params(pr.n0, e->pi, 1, &p);
        if (!sg::stir_verify(pr, p)) throw sg::SgError{SG_EVERIFY, "self-verification of the produced proof failed"};
      }
      e->status = SG_OK;
    } catch (const sg::SgError& x) {
      e->status = x.code;
      e->err = x.msg;
    } catch (const std::exception& x) {
      e->status = SG_EVERIFY;
      e->err = x.what();
    }
  }

  static void require_nonempty(const std::vector<uint8_t>& v) {
    if (v.empty()) throw sg::SgError{SG_EINVAL, "empty proof"};
  }

  static void prove(sg_ctx* c, Entry* e, bool self_verify) {
    {
      if (e->kind == SG_JOB_SHA256) {
        e->proof = sg::prove_sha256_message(c, e->input.data(), e->input.size(), e->pi, e->phi_mode, self_verify,
                                            e->digest, e->blowup);
      } else if (e->kind == SG_JOB_SHA512) {
        e->proof = sg::prove_hash_message(c, sg::sha512_hash_air(), e->input.data(), e->input.size(), e->pi,
                                          e->phi_mode, self_verify, e->digest, e->blowup);
      } else if (e->kind == SG_JOB_P256_ECDSA) {
        const uint8_t* in = e->input.data();
        e->proof = sg::prove_p256_ecdsa(c, in, in + 32, in + 64, in + 96, in + 128, e->pi, self_verify, e->blowup);
      } else if (e->kind == SG_JOB_RSA2048) {
        e->proof = prove_rsa_job(c, e->input, e->pi, e->blowup, self_verify);
      } else if (e->kind == SG_JOB_ED25519) {
        const uint8_t* in = e->input.data();
        check_ed25519_job(e->input);
        e->proof = sg::prove_ed25519(c, in, in + 32, in + 96, e->input.size() - 96, e->pi, sg::ed25519::K_FULL,
                                     self_verify, e->blowup);
      } else {
        const uint64_t n = e->input.size() / 8;
        e->proof = sg::prove_hash_rollup_host_leaves(c, (const uint64_t*)e->input.data(), n, e->pi, e->phi_mode,
                                                     self_verify);
      }
    }
  }
};

extern "C" {

int sg_server_create(sg_ctx* ctx, int n_streams, uint64_t hbm_budget_bytes, sg_server** out) {
  if (!ctx || !out || n_streams < 1 || n_streams > 256) return SG_EINVAL;
  *out = nullptr;
  sg_server* s = new sg_server;
  s->parent = ctx;
  s->group_max = ctx->stir_group;
  s->budget = hbm_budget_bytes ? hbm_budget_bytes : UINT64_MAX;
  cudaSetDevice(ctx->device);
  int prio_low = 0, prio_high = 0;
  if (cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess) {
    delete s;
    return SG_ECUDA;
  }
  for (int i = 0; i < n_streams; ++i) {
    sg_ctx* w = new sg_ctx;
    w->device = ctx->device;
    w->tw = ctx->tw;
    w->owns_tables = false;
    w->wide_merge = ctx->wide_merge;
    s->wctx.push_back(w);
    // The STIR phase (many small launches, each followed by a host round trip)
    // runs on a highest-priority stream, so its CTAs are dispatched ahead of the
    // remaining CTAs of other workers' LDE and constraint kernels.
    if (cudaStreamCreateWithFlags(&w->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithPriority(&w->stir_stream, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
        cudaEventCreateWithFlags(&w->stir_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&w->stir_out, cudaEventDisableTiming) != cudaSuccess) {
      if (!w->stream) w->stream = w->own_stream;
      sg_server_destroy(s);
      return SG_ECUDA;
    }
    w->stream = w->own_stream;
  }
  if (hbm_budget_bytes) {
    // the pool's steady-state size up front: growing it piecemeal while other
    // workers' kernels run stalls them
    try {
      sg::pool_reserve(ctx->device, hbm_budget_bytes, s->wctx[0]->stream);
    } catch (const sg::SgError&) {
      sg_server_destroy(s);
      return SG_ECUDA;
    }
  }
  for (sg_ctx* w : s->wctx) s->threads.emplace_back([s, w] { s->worker(w); });
  *out = s;
  return SG_OK;
}

void sg_server_destroy(sg_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->threads) t.join();
  for (sg_ctx* w : s->wctx) sg_ctx_destroy(w);
  delete s;
}

int sg_server_submit(sg_server* s, const sg_job* job, uint64_t* ticket) {
  if (!s || !job || !ticket) return SG_EINVAL;
  if (job->kind != SG_JOB_SHA256 && job->kind != SG_JOB_SHA512 && job->kind != SG_JOB_HASH_ROLLUP &&
      job->kind != SG_JOB_RSA2048 && job->kind != SG_JOB_P256_ECDSA && job->kind != SG_JOB_ED25519)
    return SG_EINVAL;
  if (job->kind == SG_JOB_ED25519 && job->input_len < 96) return SG_EINVAL;
  if (job->kind == SG_JOB_P256_ECDSA && job->input_len != 160) return SG_EINVAL;
  if (job->input_len && !job->input) return SG_EINVAL;
  if (job->kind == SG_JOB_RSA2048 && (job->input_len == 0 || job->input_len % 768)) return SG_EINVAL;
  if (job->blowup && (job->blowup < 2 || job->blowup > 1024 || (job->blowup & (job->blowup - 1)))) return SG_EINVAL;
  Entry e;
  e.kind = job->kind;
  e.phi_mode = job->phi_mode;
  e.blowup = job_blowup(*job);
  e.flags = job->flags;
  const size_t bytes = job->kind == SG_JOB_HASH_ROLLUP ? job->input_len * 8 : job->input_len;
  e.input.assign((const uint8_t*)job->input, (const uint8_t*)job->input + bytes);
  memcpy(e.pi, job->pi, 32);
  e.footprint = footprint_bytes(*job);
  e.t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    *ticket = s->next_ticket++;
    s->entries.emplace(*ticket, std::move(e));
    s->queue.push_back(*ticket);
  }
  s->cv_work.notify_one();
  return SG_OK;
}

int sg_server_poll(sg_server* s, uint64_t ticket) {
  if (!s) return SG_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->entries.find(ticket);
  if (it == s->entries.end()) return SG_EINVAL;
  return it->second.done ? 1 : 0;
}

namespace {

// The result of a finished job (entries locked by the caller); erases the entry
// unless the proof does not fit.
int take_result(sg_server* s, std::map<uint64_t, Entry>::iterator it, sg_job_result* res, uint8_t* proof,
                size_t cap) {
  Entry& e = it->second;
  auto ms = [](Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
  };
  memset(res, 0, sizeof *res);
  res->status = e.status;
  res->proof_len = e.proof.size();
  memcpy(res->digest, e.digest, 64);
  res->queue_ms = ms(e.t_submit, e.t_start);
  res->run_ms = ms(e.t_start, e.t_end);
  res->latency_ms = ms(e.t_submit, e.t_end);
  int rc = e.status;
  if (rc == SG_OK) {
    if (!proof || e.proof.size() > cap) return SG_ESPACE;  // entry kept: the caller may retry with a larger buffer
    memcpy(proof, e.proof.data(), e.proof.size());
  }
  s->entries.erase(it);
  return rc;
}

}  // namespace

int sg_server_wait(sg_server* s, uint64_t ticket, sg_job_result* res, uint8_t* proof, size_t cap) {
  if (!s || !res) return SG_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->entries.find(ticket);
  if (it == s->entries.end()) return SG_EINVAL;
  s->cv_done.wait(lk, [&] { return it->second.done; });
  return take_result(s, it, res, proof, cap);
}

int sg_server_wait_for(sg_server* s, uint64_t ticket, int64_t timeout_ms, sg_job_result* res, uint8_t* proof,
                       size_t cap) {
  if (!s || !res || timeout_ms < 0) return SG_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->entries.find(ticket);
  if (it == s->entries.end()) return SG_EINVAL;
  if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return it->second.done; })) {
    memset(res, 0, sizeof *res);
    res->status = SG_ETIMEDOUT;
    return SG_ETIMEDOUT;
  }
  return take_result(s, it, res, proof, cap);
}

int sg_server_cancel(sg_server* s, uint64_t ticket) {
  if (!s) return SG_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->entries.find(ticket);
  if (it == s->entries.end()) return SG_EINVAL;
  Entry& e = it->second;
  if (e.done) return 2;  // finished before the call: its result stands
  for (auto q = s->queue.begin(); q != s->queue.end(); ++q) {
    if (*q != ticket) continue;
    // queued (never started, or waiting for a retry): dropped here
    s->queue.erase(q);
    e.status = SG_ECANCELED;
    e.proof.clear();
    if (e.attempts == 0) e.t_start = Clock::now();
    e.t_end = Clock::now();
    e.done = true;
    s->cv_done.notify_all();
    return SG_OK;
  }
  e.cancel = true;  // running: the worker discards its result
  return 1;
}

int sg_server_set_retries(sg_server* s, int max_retries) {
  if (!s || max_retries < 0 || max_retries > 100) return SG_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  s->max_retries = max_retries;
  return SG_OK;
}

int sg_prove_batch(sg_ctx* ctx, const sg_job* jobs, size_t n, int n_streams, uint64_t hbm_budget_bytes,
                   uint8_t* proofs, size_t cap_per_job, sg_job_result* results) {
  if (!ctx || (n && (!jobs || !results))) return SG_EINVAL;
  sg_server* s = nullptr;
  int rc = sg_server_create(ctx, n_streams, hbm_budget_bytes, &s);
  if (rc != SG_OK) return rc;
  std::vector<uint64_t> tickets(n);
  int first_err = SG_OK;
  for (size_t i = 0; i < n; ++i) {
    rc = sg_server_submit(s, &jobs[i], &tickets[i]);
    if (rc != SG_OK) {
      tickets[i] = 0;
      results[i] = sg_job_result{};
      results[i].status = rc;
      if (first_err == SG_OK) first_err = rc;
    }
  }
  for (size_t i = 0; i < n; ++i) {
    if (!tickets[i]) continue;
    rc = sg_server_wait(s, tickets[i], &results[i], proofs ? proofs + i * cap_per_job : nullptr, cap_per_job);
    if (rc != SG_OK && first_err == SG_OK) first_err = rc;
  }
  sg_server_destroy(s);
  return first_err;
}

}  // extern "C"
