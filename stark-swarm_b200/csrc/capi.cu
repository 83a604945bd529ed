// capi.cu — extern "C" entry points declared in include/stark_gpu.h.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "context.hpp"
#include "dns.hpp"
#include "ed25519.hpp"
#include "ed25519_prover.hpp"
#include "merge.cuh"
#include "merkle.cuh"
#include "p256.hpp"
#include "p256_prover.hpp"
#include "prover.hpp"
#include "rsa_air.cuh"
#include "sha256_air.cuh"
#include "sha512_air.cuh"
#include "verifier.hpp"

struct sg_tree {
  sg::DevTree t;
  sg::DBuf buf;
};

namespace {

int fail(sg_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

template <class F>
int guarded(sg_ctx* c, F&& f) {
  if (!c) return SG_EINVAL;
  try {
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(c, SG_ECUDA, "cudaSetDevice failed");
    f();
    c->err.clear();
    return SG_OK;
  } catch (const sg::SgError& e) {
    return fail(c, e.code, e.msg);
  } catch (const std::bad_alloc&) {
    return fail(c, SG_ENOMEM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(c, SG_EINVAL, e.what());
  }
}

template <class F>
int host_guarded(F&& f) {
  try {
    f();
    return SG_OK;
  } catch (const sg::SgError& e) {
    return e.code;
  } catch (const std::bad_alloc&) {
    return SG_ENOMEM;
  }
}
bool ed_args(const uint8_t* pub, const uint8_t* sig, const uint8_t* msg, size_t len) {
  return pub && sig && (msg || len == 0);
}

// A caller buffer on the device is used in place; a host buffer is staged.
struct In {
  const uint64_t* d = nullptr;
  sg::DBuf stage;
  In(const uint64_t* p, size_t elems, cudaStream_t s) {
    if (elems == 0 || sg::is_device_ptr(p)) {
      d = p;
      return;
    }
    stage.alloc(elems, s);
    sg::cuda_check(cudaMemcpyAsync(stage.p, p, elems * 8, cudaMemcpyHostToDevice, s), "h2d");
    d = stage.p;
  }
};
struct Out {
  uint64_t* user;
  uint64_t* d = nullptr;
  size_t elems;
  bool host = false;
  sg::DBuf stage;
  cudaStream_t s;
  Out(uint64_t* p, size_t n, cudaStream_t st) : user(p), elems(n), s(st) {
    if (n == 0 || sg::is_device_ptr(p)) {
      d = p;
      return;
    }
    host = true;
    stage.alloc(n, s);
    d = stage.p;
  }
  void finish() {
    if (host) sg::cuda_check(cudaMemcpyAsync(user, d, elems * 8, cudaMemcpyDeviceToHost, s), "d2h");
    sg::cuda_check(cudaStreamSynchronize(s), "sync");
  }
};

}  // namespace

namespace sg {

// Pinned staging buffers are recycled process-wide: a context returns its buffer
// when it is destroyed (server workers come and go with each batch), so page
// locking happens once per peak concurrency, not once per worker.
namespace {
struct PinnedPool {
  std::mutex mu;
  std::vector<std::pair<void*, size_t>> free;
};
PinnedPool& pinned_pool() {
  static PinnedPool* p = new PinnedPool;  // kept for the process
  return *p;
}
}  // namespace

void pinned_release(sg_ctx* c) {
  if (!c->pinned) return;
  PinnedPool& P = pinned_pool();
  std::lock_guard<std::mutex> g(P.mu);
  P.free.push_back({c->pinned, c->pinned_bytes});
  c->pinned = nullptr;
  c->pinned_bytes = 0;
}

void* pinned_host(sg_ctx* c, size_t bytes) {
  if (c->pinned_bytes >= bytes) return c->pinned;
  cuda_check(cudaStreamSynchronize(c->stream), "sync");  // no copy from the old buffer in flight
  pinned_release(c);
  {
    PinnedPool& P = pinned_pool();
    std::lock_guard<std::mutex> g(P.mu);
    size_t best = P.free.size();
    for (size_t i = 0; i < P.free.size(); ++i)
      if (P.free[i].second >= bytes && (best == P.free.size() || P.free[i].second < P.free[best].second)) best = i;
    if (best < P.free.size()) {
      c->pinned = P.free[best].first;
      c->pinned_bytes = P.free[best].second;
      P.free.erase(P.free.begin() + best);
      return c->pinned;
    }
  }
  void* p = nullptr;
  cuda_check(cudaHostAlloc(&p, bytes, cudaHostAllocDefault), "pinned host allocation");
  c->pinned = p;
  c->pinned_bytes = bytes;
  return p;
}

void pool_reserve(int device, uint64_t bytes, cudaStream_t s) {
  cuda_check(cudaSetDevice(device), "set device");
  cudaMemPool_t pool;
  cuda_check(cudaDeviceGetDefaultMemPool(&pool, device), "memory pool");
  uint64_t reserved = 0;
  cuda_check(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved), "memory pool");
  if (reserved >= bytes) return;
  size_t free_b = 0, total_b = 0;
  cuda_check(cudaMemGetInfo(&free_b, &total_b), "memory info");
  const uint64_t margin = 2ull << 30;
  if (free_b <= margin) return;
  const uint64_t want = std::min<uint64_t>(bytes - reserved, free_b - margin);
  void* p = nullptr;
  if (cudaMallocAsync(&p, want, s) != cudaSuccess) {
    cudaGetLastError();  // nothing reserved; proofs grow the pool as they go
    return;
  }
  cuda_check(cudaFreeAsync(p, s), "free");
  cuda_check(cudaStreamSynchronize(s), "sync");
}

}  // namespace sg

extern "C" {

int sg_ctx_create(int device, sg_ctx** out) {
  if (!out) return SG_EINVAL;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return SG_ECUDA;
  }
  if (device < 0 || device >= n) return SG_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return SG_ECUDA;
  sg_ctx* c = new sg_ctx;
  c->device = device;
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return SG_ECUDA;
  }
  c->stream = c->own_stream;
  if (sg::ntt_tables_init(&c->tw) != cudaSuccess) {
    cudaStreamDestroy(c->own_stream);
    delete c;
    return SG_ECUDA;
  }
  // Keep freed pool memory cached, so repeated proofs reuse it without cudaMalloc.
  // Never let the pool satisfy an allocation on one stream with a block freed on
  // another by making the first stream wait for the second: contexts proving
  // concurrently (a Merkle commitment beside a STIR proof, server workers) would
  // be serialised behind each other. The pool grows instead.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    int no = 0;
    cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
  }
  *out = c;
  return SG_OK;
}

void sg_ctx_destroy(sg_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->owns_tables) sg::ntt_tables_free(&c->tw);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
  }
  if (c->shift_tab) cudaFree(c->shift_tab);
  if (c->stir_stream) {
    cudaStreamSynchronize(c->stir_stream);
    cudaStreamDestroy(c->stir_stream);
  }
  if (c->stir_in) cudaEventDestroy(c->stir_in);
  if (c->stir_out) cudaEventDestroy(c->stir_out);
  sg::pinned_release(c);
  delete c;
}

int sg_ctx_set_stream(sg_ctx* c, void* stream) {
  if (!c) return SG_EINVAL;
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return SG_OK;
}

const char* sg_last_error(const sg_ctx* c) { return c ? c->err.c_str() : "null context"; }

int sg_ctx_set_option(sg_ctx* c, int option, int64_t value) {
  if (!c) return SG_EINVAL;
  if (option == SG_OPT_WIDE_MERGE) {
    if (value < SG_WIDE_MERGE_AUTO || value > SG_WIDE_MERGE_COSETS) return SG_EINVAL;
    c->wide_merge = (int)value;
    return SG_OK;
  }
  if (option == SG_OPT_STIR_GROUP) {
    if (value < 1 || value > 64) return SG_EINVAL;
    c->stir_group = (int)value;
    return SG_OK;
  }
  return SG_EINVAL;
}

int sg_hash_bytes(void) { return kc::kHashBytes; }

int sg_ntt_set_split(size_t log_n, int padded, int log_n1) {
  if (log_n < 13 || log_n > 24) return SG_EINVAL;
  if (log_n1 != 0 && (log_n1 < std::max<int>(1, (int)log_n - 12) || log_n1 > std::min<int>(12, (int)log_n - 1)))
    return SG_EINVAL;
  sg::ntt_set_split((int)log_n, padded != 0, log_n1);
  return SG_OK;
}

int sg_ntt_autotune(sg_ctx* c, size_t n_cols, size_t log_n, int inverse, size_t n_valid, int* best_log_n1) {
  return guarded(c, [&] {
    sg::require(log_n >= 13 && log_n <= 24 && n_cols > 0, "ntt_autotune: sizes 2^13 .. 2^24 (two passes) only");
    const uint64_t N = 1ull << log_n;
    if (n_valid == 0 || n_valid > N) n_valid = N;
    const bool padded = n_valid < N;
    // enough columns to fill the GPU (2^26 elements), at most the caller's
    const uint64_t cols = std::min<uint64_t>(n_cols, std::max<uint64_t>(1, (1ull << 26) >> log_n));
    cudaStream_t s = c->stream;
    sg::DBuf in(cols * N, s), out(cols * N, s), scratch(sg::ntt_scratch_elems(cols, (int)log_n), s);
    sg::cuda_check(cudaMemsetAsync(in.p, 0, cols * N * 8, s), "memset");  // the timing is data-independent
    cudaEvent_t e0, e1;
    sg::cuda_check(cudaEventCreate(&e0), "event");
    sg::cuda_check(cudaEventCreate(&e1), "event");
    const int lo = std::max<int>(1, (int)log_n - 12), hi = std::min<int>(12, (int)log_n - 1);
    const int prior = sg::ntt_split((int)log_n, padded);
    int best = prior;
    float best_ms = 1e30f;
    try {
      for (int l1 = lo; l1 <= hi; ++l1) {
        sg::ntt_set_split((int)log_n, padded, l1);
        auto run = [&] {
          sg::cuda_check(sg::ntt_batch(c->tw, in.p, out.p, (uint32_t)cols, N, N, (int)log_n, inverse != 0, n_valid,
                                       scratch.p, s),
                         "ntt");
        };
        run();  // warm-up
        float ms = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
          sg::cuda_check(cudaEventRecord(e0, s), "event");
          run();
          sg::cuda_check(cudaEventRecord(e1, s), "event");
          sg::cuda_check(cudaEventSynchronize(e1), "sync");
          float t = 0;
          sg::cuda_check(cudaEventElapsedTime(&t, e0, e1), "elapsed");
          ms = std::min(ms, t);
        }
        if (ms < best_ms) {
          best_ms = ms;
          best = l1;
        }
      }
    } catch (...) {
      sg::ntt_set_split((int)log_n, padded, prior);
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    sg::ntt_set_split((int)log_n, padded, best);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (best_log_n1) *best_log_n1 = best;
  });
}

int sg_pool_reserve(sg_ctx* c, uint64_t bytes) {
  return guarded(c, [&] { sg::pool_reserve(c->device, bytes, c->stream); });
}

uint64_t sg_kernel_launches(const sg_ctx*) { return sg::g_kernel_launches.load(); }

int sg_profile_enable(int on) {
  sg::Profiler::get().enable(on != 0);
  return SG_OK;
}

int sg_profile_read(sg_profile_entry* out, size_t cap, size_t* n) {
  std::vector<sg::ProfStat> st = sg::Profiler::get().read();
  if (n) *n = st.size();
  for (size_t i = 0; i < st.size() && i < cap && out; ++i) {
    memset(out[i].name, 0, sizeof out[i].name);
    strncpy(out[i].name, st[i].name.c_str(), sizeof out[i].name - 1);
    out[i].launches = st[i].launches;
    out[i].total_ms = st[i].total_ms;
  }
  return SG_OK;
}

void sg_profile_reset(void) { sg::Profiler::get().reset(); }

int sg_ntt(sg_ctx* c, const uint64_t* in, uint64_t* out, size_t n_cols, size_t log_n, int inverse) {
  return guarded(c, [&] {
    sg::require(in && out && n_cols > 0 && n_cols < (1u << 31), "ntt: bad buffers or column count");
    sg::require(log_n <= (size_t)sg::kMaxLogN, "ntt: log_n must be <= 28");
    const size_t n = size_t(1) << log_n, total = n_cols * n;
    In di(in, total, c->stream);
    Out dout(out, total, c->stream);
    sg::DBuf scratch(sg::ntt_scratch_elems(n_cols, (int)log_n), c->stream);
    sg::cuda_check(sg::ntt_batch(c->tw, di.d, dout.d, (uint32_t)n_cols, n, n, (int)log_n, inverse != 0, n,
                                 scratch.p, c->stream),
                   "ntt");
    dout.finish();
  });
}

int sg_lde(sg_ctx* c, const uint64_t* trace, size_t w, size_t n_trace, size_t blowup, uint64_t shift,
           uint64_t* out) {
  return guarded(c, [&] {
    sg::require(trace && out, "lde: null buffer");
    sg::require(w > 0 && n_trace > 0 && blowup > 0, "lde: empty input");
    Out dout(out, w * n_trace * blowup, c->stream);
    if (sg::is_device_ptr(trace)) {
      sg::lde_device(c, trace, w, n_trace, blowup, shift, dout.d);
    } else {
      sg::lde_from_host(c, trace, w, n_trace, blowup, shift, dout.d);  // copy overlapped with the transform
    }
    dout.finish();
  });
}

int sg_merge(sg_ctx* c, int air, const uint64_t* lde, size_t w, size_t n_trace, size_t blowup,
             const uint64_t* lambdas, size_t k, int phi_mode, uint64_t* c_eval) {
  return guarded(c, [&] {
    sg::require(lde && lambdas && c_eval, "merge: null buffer");
    sg::require(n_trace > 0 && blowup > 0, "merge: empty input");
    const size_t n = n_trace * blowup;
    std::vector<uint64_t> lam(lambdas, lambdas + k);  // lambdas are read on the host
    In di(lde, w * n, c->stream);
    Out dout(c_eval, n, c->stream);
    sg::merge_device(c, air, di.d, w, n_trace, blowup, lam.data(), k, phi_mode, dout.d);
    dout.finish();
  });
}

int sg_merge_sha256(sg_ctx* c, const uint64_t* lde, size_t n_trace, size_t blowup, const uint64_t* lambdas,
                    size_t n_blocks, int phi_mode, uint64_t* c_eval) {
  return guarded(c, [&] {
    sg::require(lde && lambdas && c_eval, "merge_sha256: null buffer");
    sg::require(n_trace > 0 && blowup > 0 && n_blocks > 0, "merge_sha256: empty input");
    const size_t n = n_trace * blowup;
    std::vector<uint64_t> lam(lambdas, lambdas + sg::sha::NUM_CONSTRAINTS);
    In di(lde, (size_t)sg::sha::WIDTH * n, c->stream);
    Out dout(c_eval, n, c->stream);
    sg::merge_device(c, SG_AIR_SHA256, di.d, sg::sha::WIDTH, n_trace, blowup, lam.data(), lam.size(), phi_mode,
                     dout.d, n_blocks);
    dout.finish();
  });
}

int sg_sha256_trace(const uint8_t* msg, size_t len, uint64_t* trace, size_t cap, size_t* height, size_t* n_blocks,
                    uint8_t digest[32]) {
  if ((!msg && len) || !height || !n_blocks || !digest) return SG_EINVAL;
  try {
    std::vector<sg::sha::BlockWitness> wit;
    uint8_t dg[32];
    const uint64_t h = sg::sha256_witness(msg, len, &wit, dg);
    *height = (size_t)h;
    *n_blocks = wit.size();
    memcpy(digest, dg, 32);
    if (!trace || (uint64_t)sg::sha::WIDTH * h > cap) return SG_ESPACE;
    sg::sha256_fill_host(wit.data(), wit.size(), h, trace);
    return SG_OK;
  } catch (const std::bad_alloc&) {
    return SG_ENOMEM;
  }
}

int sg_sha256_trace_gpu(sg_ctx* c, const uint8_t* msg, size_t len, uint64_t* trace, size_t cap, size_t* height,
                        size_t* n_blocks, uint8_t digest[32]) {
  return guarded(c, [&] {
    sg::require((msg || !len) && height && n_blocks && digest, "sha256_trace_gpu: null argument");
    std::vector<sg::sha::BlockWitness> wit;
    const uint64_t h = sg::sha256_witness(msg, len, &wit, digest);
    *height = (size_t)h;
    *n_blocks = wit.size();
    const uint64_t cells = (uint64_t)sg::sha::WIDTH * h;
    if (!trace || cells > cap) throw sg::SgError{SG_ESPACE, "sha256_trace_gpu: trace buffer too small"};
    Out dout(trace, cells, c->stream);
    sg::DBuf d_wit((wit.size() * sizeof(sg::sha::BlockWitness) + 7) / 8, c->stream);
    sg::cuda_check(cudaMemcpyAsync(d_wit.p, wit.data(), wit.size() * sizeof(sg::sha::BlockWitness),
                                   cudaMemcpyHostToDevice, c->stream), "h2d");
    sg::cuda_check(sg::sha256_expand((const sg::sha::BlockWitness*)d_wit.p, wit.size(), h, dout.d, c->stream),
                   "sha256_expand");
    dout.finish();
  });
}

int sg_prove_sha256(sg_ctx* c, const uint8_t* msg, size_t len, const uint8_t fs_binding[32], int phi_mode,
                    uint8_t* proof, size_t cap, size_t* len_out, uint8_t digest[32]) {
  return guarded(c, [&] {
    sg::require((msg || !len) && fs_binding && len_out && digest, "prove_sha256: null argument");
    std::vector<uint8_t> b = sg::prove_sha256_message(c, msg, len, fs_binding, phi_mode, true, digest);
    *len_out = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_sha256: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

int sg_merge_sha512(sg_ctx* c, const uint64_t* lde, size_t n_trace, size_t blowup, const uint64_t* lambdas,
                    size_t n_blocks, int phi_mode, uint64_t* c_eval) {
  return guarded(c, [&] {
    sg::require(lde && lambdas && c_eval, "merge_sha512: null buffer");
    sg::require(n_trace > 0 && blowup > 0 && n_blocks > 0, "merge_sha512: empty input");
    const size_t n = n_trace * blowup;
    In di(lde, (size_t)sg::sha512::WIDTH * n, c->stream);
    Out dout(c_eval, n, c->stream);
    sg::merge_hash_device(c, sg::sha512_hash_air(), di.d, n_trace, blowup, lambdas, phi_mode, dout.d, n_blocks);
    dout.finish();
  });
}

int sg_sha512_trace(const uint8_t* msg, size_t len, uint64_t* trace, size_t cap, size_t* height, size_t* n_blocks,
                    uint8_t digest[64]) {
  if ((!msg && len) || !height || !n_blocks || !digest) return SG_EINVAL;
  try {
    std::vector<sg::sha512::BlockWitness> wit;
    uint8_t dg[64];
    const uint64_t h = sg::sha512_witness(msg, len, &wit, dg);
    *height = (size_t)h;
    *n_blocks = wit.size();
    memcpy(digest, dg, 64);
    if (!trace || (uint64_t)sg::sha512::WIDTH * h > cap) return SG_ESPACE;
    sg::sha512_fill_host(wit.data(), wit.size(), h, trace);
    return SG_OK;
  } catch (const std::bad_alloc&) {
    return SG_ENOMEM;
  }
}

int sg_sha512_trace_gpu(sg_ctx* c, const uint8_t* msg, size_t len, uint64_t* trace, size_t cap, size_t* height,
                        size_t* n_blocks, uint8_t digest[64]) {
  return guarded(c, [&] {
    sg::require((msg || !len) && height && n_blocks && digest, "sha512_trace_gpu: null argument");
    std::vector<sg::sha512::BlockWitness> wit;
    const uint64_t h = sg::sha512_witness(msg, len, &wit, digest);
    *height = (size_t)h;
    *n_blocks = wit.size();
    const uint64_t cells = (uint64_t)sg::sha512::WIDTH * h;
    if (!trace || cells > cap) throw sg::SgError{SG_ESPACE, "sha512_trace_gpu: trace buffer too small"};
    Out dout(trace, cells, c->stream);
    sg::DBuf d_wit((wit.size() * sizeof(sg::sha512::BlockWitness) + 7) / 8, c->stream);
    sg::cuda_check(cudaMemcpyAsync(d_wit.p, wit.data(), wit.size() * sizeof(sg::sha512::BlockWitness),
                                   cudaMemcpyHostToDevice, c->stream), "h2d");
    sg::cuda_check(sg::sha512_expand((const sg::sha512::BlockWitness*)d_wit.p, wit.size(), h, dout.d, c->stream),
                   "sha512_expand");
    dout.finish();
  });
}

int sg_prove_sha512(sg_ctx* c, const uint8_t* msg, size_t len, const uint8_t fs_binding[32], int phi_mode,
                    uint8_t* proof, size_t cap, size_t* len_out, uint8_t digest[64]) {
  return guarded(c, [&] {
    sg::require((msg || !len) && fs_binding && len_out && digest, "prove_sha512: null argument");
    std::vector<uint8_t> b =
        sg::prove_hash_message(c, sg::sha512_hash_air(), msg, len, fs_binding, phi_mode, true, digest);
    *len_out = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_sha512: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

// ------------------------------------------------------------------ RSA-2048
int sg_rsa2048_em(const uint8_t* msg, size_t len, uint8_t em[256]) {
  if ((!msg && len) || !em) return SG_EINVAL;
  return host_guarded([&] { sg::rsa::em_encode(msg, len, em); });
}

int sg_rsa2048_verify(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t em[256]) {
  if (!n_be || !s_be || !em) return 0;
  try {
    return sg::rsa::verify_native(n_be, s_be, em) ? 1 : 0;
  } catch (...) {
    return 0;
  }
}

int sg_rsa2048_pi_record(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t* msg, size_t len,
                         const uint8_t em[256], uint8_t out[32]) {
  if (!n_be || !s_be || (!msg && len) || !em || !out) return SG_EINVAL;
  return host_guarded([&] { sg::rsa::pi_record(n_be, s_be, msg, len, em, out); });
}

int sg_rsa2048_pi_stacked(const uint8_t n_be[256], size_t n_records, const uint8_t* ems, uint8_t out[32]) {
  if (!n_be || (!ems && n_records) || !out) return SG_EINVAL;
  return host_guarded([&] { sg::rsa::pi_stacked(n_be, n_records, ems, out); });
}

int sg_rsa2048_trace(const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be, size_t n_records,
                     uint64_t* trace, size_t cap) {
  if (!n_be || !s_be || !em_be || n_records == 0) return SG_EINVAL;
  try {
    std::vector<sg::rsa::RecordW> recs;
    std::vector<sg::rsa::RowW> rows;
    sg::rsa_witnesses(n_be, s_be, em_be, n_records, &recs, &rows);
    if (!trace || (uint64_t)n_records * sg::rsa::WIDTH * sg::rsa::N_TRACE > cap) return SG_ESPACE;
    sg::rsa::expand_host(recs.data(), rows.data(), n_records, trace);
    return SG_OK;
  } catch (const sg::SgError& e) {
    return e.code;
  } catch (const std::bad_alloc&) {
    return SG_ENOMEM;
  }
}

int sg_rsa2048_trace_gpu(sg_ctx* c, const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be,
                         size_t n_records, uint64_t* trace, size_t cap) {
  return guarded(c, [&] {
    sg::require(n_be && s_be && em_be && n_records > 0, "rsa2048_trace_gpu: null argument");
    std::vector<sg::rsa::RecordW> recs;
    std::vector<sg::rsa::RowW> rows;
    sg::rsa_witnesses(n_be, s_be, em_be, n_records, &recs, &rows);
    const uint64_t cells = (uint64_t)n_records * sg::rsa::WIDTH * sg::rsa::N_TRACE;
    if (!trace || cells > cap) throw sg::SgError{SG_ESPACE, "rsa2048_trace_gpu: trace buffer too small"};
    Out dout(trace, cells, c->stream);
    const size_t rb = recs.size() * sizeof(sg::rsa::RecordW), wb = rows.size() * sizeof(sg::rsa::RowW);
    sg::DBuf d_wit((rb + wb + 7) / 8, c->stream);
    uint8_t* base = (uint8_t*)d_wit.p;
    sg::cuda_check(cudaMemcpyAsync(base, recs.data(), rb, cudaMemcpyHostToDevice, c->stream), "h2d");
    sg::cuda_check(cudaMemcpyAsync(base + rb, rows.data(), wb, cudaMemcpyHostToDevice, c->stream), "h2d");
    sg::cuda_check(sg::rsa_expand((const sg::rsa::RecordW*)base, (const sg::rsa::RowW*)(base + rb), n_records,
                                  dout.d, c->stream),
                   "rsa_expand");
    dout.finish();
  });
}

int sg_merge_rsa2048(sg_ctx* c, const uint64_t* lde, size_t n_records, size_t n_trace, size_t blowup,
                     uint64_t* c_eval) {
  return guarded(c, [&] {
    sg::require(lde && c_eval && n_records > 0 && n_records <= 65535, "merge_rsa2048: bad argument");
    sg::require(n_trace >= 2 && (n_trace & (n_trace - 1)) == 0 && blowup >= 4 && (blowup & (blowup - 1)) == 0,
                "merge_rsa2048: n_trace and blowup must be powers of 2 (blowup >= 4)");
    const size_t n = n_trace * blowup;
    unsigned ln = 0;
    while ((size_t(1) << ln) < n) ++ln;
    sg::require(ln <= sg::kMaxLogN, "merge_rsa2048: domain larger than 2^28");
    cudaStream_t s = c->stream;
    In di(lde, n_records * sg::rsa::WIDTH * n, s);
    Out dout(c_eval, n, s);
    sg::DBuf phi(n, s), part(n_records > 1 ? n_records * n : 0, s), scratch(sg::ntt_scratch_elems(1, ln), s);
    sg::cuda_check(sg::rsa_phi(di.d, n_records, n_trace, blowup, part.p, phi.p, s), "rsa phi");
    sg::cuda_check(sg::ntt_batch(c->tw, phi.p, phi.p, 1, n, n, ln, true, n, scratch.p, s), "intt");
    sg::cuda_check(sg::quotient_zh(phi.p, n, n_trace, dout.d, s), "quotient");
    sg::cuda_check(sg::ntt_batch(c->tw, dout.d, dout.d, 1, n, n, ln, false, n - n_trace, scratch.p, s), "ntt");
    dout.finish();
  });
}

int sg_prove_rsa2048(sg_ctx* c, const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be, size_t n_records,
                     const uint8_t pi[32], uint8_t* proof, size_t cap, size_t* len) {
  return guarded(c, [&] {
    sg::require(n_be && s_be && em_be && pi && len, "prove_rsa2048: null argument");
    std::vector<uint8_t> b = sg::prove_rsa2048(c, n_be, s_be, em_be, n_records, pi, true);
    *len = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_rsa2048: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

// ------------------------------------------------------------------ P-256 ECDSA
int sg_p256_layout(uint32_t* width, uint32_t* n_gadgets, uint32_t* n_constraints, uint32_t* table, size_t cap,
                   uint32_t tail[18]) {
  if (!width || !n_gadgets || !n_constraints) return SG_EINVAL;
  try {
    const sg::p256::Layout& L = sg::p256::layout();
    *width = L.width;
    *n_gadgets = (uint32_t)L.table.size();
    *n_constraints = L.n_constraints;
    if (tail) memcpy(tail, L.tail, sizeof L.tail);
    if (table) {
      if (cap < L.table.size()) return SG_ESPACE;
      memcpy(table, L.table.data(), L.table.size() * sizeof(sg::p256::Gadget));
    }
    return SG_OK;
  } catch (const sg::SgError& e) {
    return e.code;
  }
}

int sg_p256_u_bits(const uint8_t digest[32], const uint8_t r[32], const uint8_t s[32], uint8_t u1[256],
                   uint8_t u2[256]) {
  if (!digest || !r || !s || !u1 || !u2) return SG_EINVAL;
  try {
    sg::p256::u_bits(digest, r, s, u1, u2);
    return SG_OK;
  } catch (const sg::SgError& e) {
    return e.code;
  }
}

int sg_p256_ecdsa_pi(const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32], const uint8_t s[32],
                     const uint8_t digest[32], uint8_t out[32]) {
  if (!qx || !qy || !r || !s || !digest || !out) return SG_EINVAL;
  return host_guarded([&] { sg::p256::pi_hash(qx, qy, r, s, digest, out); });
}

int sg_p256_chain_trace(const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits, const uint8_t bx[32],
                        const uint8_t by[32], const uint8_t* b_bits, size_t k, uint64_t* trace, size_t cap) {
  if (!ax || !ay || !a_bits || !bx || !by || !b_bits || k < 2 || (k & (k - 1)) || k > 65536) return SG_EINVAL;
  try {
    std::vector<sg::p256::RowW> rows(k);
    std::vector<sg::p256::GadgetW> gw(k * sg::p256::layout().table.size());
    uint32_t rproj[6][sg::p256::NL];
    sg::p256::chain_witness(ax, ay, a_bits, bx, by, b_bits, k, rows.data(), gw.data(), rproj);
    if (!trace || (uint64_t)sg::p256::layout().width * k > cap) return SG_ESPACE;
    sg::p256::expand_host(rows.data(), gw.data(), rproj, k, trace);
    return SG_OK;
  } catch (const sg::SgError& e) {
    return e.code;
  } catch (const std::bad_alloc&) {
    return SG_ENOMEM;
  }
}

int sg_p256_chain_trace_gpu(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                            const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, size_t k,
                            uint64_t* trace, size_t cap) {
  return guarded(c, [&] {
    sg::require(ax && ay && a_bits && bx && by && b_bits, "p256_chain_trace_gpu: null argument");
    const uint64_t cells = (uint64_t)sg::p256::layout().width * k;
    if (!trace || cells > cap) throw sg::SgError{SG_ESPACE, "p256_chain_trace_gpu: trace buffer too small"};
    Out dout(trace, cells, c->stream);
    sg::p256_trace_device(c, ax, ay, a_bits, bx, by, b_bits, k, dout.d);
    dout.finish();
  });
}

int sg_merge_p256_ecdsa(sg_ctx* c, const uint64_t* lde, size_t n_trace, size_t blowup, uint64_t* c_eval) {
  return guarded(c, [&] {
    sg::require(lde && c_eval && n_trace >= 2 && blowup >= 1, "merge_p256_ecdsa: bad argument");
    const size_t n = n_trace * blowup;
    In di(lde, (size_t)sg::p256::layout().width * n, c->stream);
    Out dout(c_eval, n, c->stream);
    sg::p256_merge_device(c, di.d, n_trace, blowup, dout.d);
    dout.finish();
  });
}

int sg_prove_p256_chains(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                         const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, size_t k,
                         const uint8_t pi[32], uint8_t* proof, size_t cap, size_t* len) {
  return guarded(c, [&] {
    sg::require(ax && ay && a_bits && bx && by && b_bits && pi && len, "prove_p256_chains: null argument");
    std::vector<uint8_t> b = sg::prove_p256_chains(c, ax, ay, a_bits, bx, by, b_bits, k, pi, true);
    *len = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_p256_chains: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

int sg_prove_p256_ecdsa(sg_ctx* c, const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32],
                        const uint8_t s[32], const uint8_t digest[32], const uint8_t pi[32], uint8_t* proof,
                        size_t cap, size_t* len) {
  return guarded(c, [&] {
    sg::require(qx && qy && r && s && digest && pi && len, "prove_p256_ecdsa: null argument");
    std::vector<uint8_t> b = sg::prove_p256_ecdsa(c, qx, qy, r, s, digest, pi, true);
    *len = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_p256_ecdsa: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

// ------------------------------------------------------------------ Ed25519
int sg_ed25519_layout(uint32_t k_scalar, size_t msg_len, uint32_t* width, uint32_t* height, uint32_t* n_constraints,
                      uint32_t rows[11]) {
  if (!width || !height || !n_constraints) return SG_EINVAL;
  return host_guarded([&] {
    const sg::ed25519::Layout L = sg::ed25519::make_layout(64 + (uint64_t)msg_len, k_scalar);
    *width = L.width;
    *height = L.height;
    *n_constraints = L.n_constraints;
    if (rows) {
      const uint32_t r[11] = {L.k_hash,   L.reduce_row,   L.decomp_R_row, L.decomp_A_row, L.sB_first, L.kA_first,
                              L.residual_row, L.dbl_row[0], L.dbl_row[1], L.dbl_row[2], L.result_row};
      memcpy(rows, r, sizeof r);
    }
  });
}

int sg_ed25519_program(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                       uint32_t k_scalar, uint64_t* recs, size_t cap_recs, size_t* n_recs, uint64_t* pairs,
                       size_t cap_pairs, size_t* n_pairs) {
  if (!ed_args(pub, sig, msg, msg_len) || !n_recs || !n_pairs) return SG_EINVAL;
  return host_guarded([&] {
    sg::ed25519::Witness w;
    sg::ed25519::build_witness(pub, sig, msg, msg_len, k_scalar, &w);
    const auto& P = w.prog;
    *n_recs = P.blocks.size();
    *n_pairs = P.pairs.size() / 2;
    if (recs) {
      if (cap_recs < P.blocks.size()) throw sg::SgError{SG_ESPACE, "ed25519_program: record buffer too small"};
      for (size_t i = 0; i < P.blocks.size(); ++i) {
        const sg::ed25519::Block& b = P.blocks[i];
        uint64_t* r = recs + 16 * i;
        for (int j = 0; j < 16; ++j) r[j] = ~0ull;
        r[0] = b.gate;
        for (int j = 0; j < 3; ++j) r[1 + j] = b.g[j] == ~0u ? ~0ull : b.g[j];
        r[4] = b.kind;
        static const int n_params[11] = {0, 1, 8, 3, 5, 5, 6, 4, 2, 2, 2};
        for (int j = 0; j < n_params[b.kind]; ++j) r[5 + j] = b.p[j];
      }
    }
    if (pairs) {
      if (cap_pairs < P.pairs.size() / 2) throw sg::SgError{SG_ESPACE, "ed25519_program: pair buffer too small"};
      memcpy(pairs, P.pairs.data(), P.pairs.size() * 8);
    }
  });
}

int sg_ed25519_trace(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                     uint32_t k_scalar, uint64_t* trace, size_t cap) {
  if (!ed_args(pub, sig, msg, msg_len)) return SG_EINVAL;
  return host_guarded([&] {
    sg::ed25519::Witness w;
    sg::ed25519::build_witness(pub, sig, msg, msg_len, k_scalar, &w);
    if (!trace || (uint64_t)w.L.width * w.L.height > cap)
      throw sg::SgError{SG_ESPACE, "ed25519_trace: trace buffer too small"};
    sg::ed25519::expand_host(w, trace);
  });
}

int sg_ed25519_trace_gpu(sg_ctx* c, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg,
                         size_t msg_len, uint32_t k_scalar, uint64_t* trace, size_t cap) {
  return guarded(c, [&] {
    sg::require(ed_args(pub, sig, msg, msg_len), "ed25519_trace_gpu: null argument");
    sg::ed25519::Witness w;
    sg::ed25519::build_witness(pub, sig, msg, msg_len, k_scalar, &w);
    const uint64_t cells = (uint64_t)w.L.width * w.L.height;
    if (!trace || cells > cap) throw sg::SgError{SG_ESPACE, "ed25519_trace_gpu: trace buffer too small"};
    Out dout(trace, cells, c->stream);
    sg::ed25519_trace_device(c, w, dout.d);
    dout.finish();
  });
}

int sg_merge_ed25519(sg_ctx* c, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                     uint32_t k_scalar, const uint64_t* lde, size_t blowup, uint64_t* c_eval) {
  return guarded(c, [&] {
    sg::require(ed_args(pub, sig, msg, msg_len) && lde && c_eval, "merge_ed25519: null argument");
    sg::check_blowup(blowup);
    sg::ed25519::Witness w;
    sg::ed25519::build_witness(pub, sig, msg, msg_len, k_scalar, &w);
    const size_t n = (size_t)w.L.height * blowup;
    In di(lde, (size_t)w.L.width * n, c->stream);
    Out dout(c_eval, n, c->stream);
    sg::ed25519_merge_device(c, w, di.d, blowup, dout.d);
    dout.finish();
  });
}

int sg_prove_ed25519(sg_ctx* c, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                     const uint8_t fs_binding[32], uint32_t k_scalar, size_t blowup, uint8_t* proof, size_t cap,
                     size_t* len) {
  return guarded(c, [&] {
    sg::require(ed_args(pub, sig, msg, msg_len) && fs_binding && len, "prove_ed25519: null argument");
    std::vector<uint8_t> b = sg::prove_ed25519(c, pub, sig, msg, msg_len, fs_binding, k_scalar, true, blowup);
    *len = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_ed25519: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

int sg_ed25519_verify(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len) {
  if (!ed_args(pub, sig, msg, msg_len)) return SG_EINVAL;
  bool ok = false;
  const int rc = host_guarded([&] { ok = sg::ed25519::verify(pub, sig, msg, msg_len); });
  return rc != SG_OK ? rc : ok ? 1 : 0;
}

int sg_ed25519_pi_hash(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, size_t msg_len,
                       const uint8_t fs_binding[32], const uint8_t merkle_root[32], const uint8_t root_f0[32],
                       uint8_t out[32]) {
  if (!ed_args(pub, sig, msg, msg_len) || !fs_binding || !merkle_root || !root_f0 || !out) return SG_EINVAL;
  return host_guarded([&] { sg::ed25519::pi_hash(pub, sig, msg, msg_len, fs_binding, merkle_root, root_f0, out); });
}

int sg_prove_zsk_ksk_binding_v2(sg_ctx* c, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg,
                                size_t msg_len, const uint8_t fs_binding[32], const uint8_t merkle_root[32],
                                uint32_t k_scalar, uint8_t* proof, size_t cap, size_t* len, uint8_t pi_hash[32]) {
  return guarded(c, [&] {
    sg::require(ed_args(pub, sig, msg, msg_len) && fs_binding && merkle_root && len && pi_hash,
                "prove_zsk_ksk_binding_v2: null argument");
    sg::require(SG_HASH_BYTES == 32, "prove_zsk_ksk_binding_v2: the bundle binds 32-byte roots (SHA3-256 profile)");
    if (!sg::ed25519::verify(pub, sig, msg, msg_len))
      throw sg::SgError{SG_EVERIFY, "prove_zsk_ksk_binding_v2: native Ed25519 verification failed"};
    std::vector<uint8_t> b =
        sg::prove_ed25519(c, pub, sig, msg, msg_len, fs_binding, k_scalar, true, sg::ed25519::BLOWUP);
    *len = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_zsk_ksk_binding_v2: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
    sg::ed25519::pi_hash(pub, sig, msg, msg_len, fs_binding, merkle_root, b.data(), pi_hash);
  });
}

int sg_dns_record_leaves(const uint8_t* canon, const size_t* offsets, size_t n, const uint8_t salt[16],
                         uint8_t* out) {
  if (!offsets || !salt || (n && (!canon || !out))) return SG_EINVAL;
  for (size_t i = 0; i < n; ++i)
    if (offsets[i + 1] < offsets[i]) return SG_EINVAL;
  return host_guarded([&] { sg::dns_record_leaves(canon, offsets, n, salt, out); });
}

int sg_dns_merkle_root(const uint8_t* leaves, size_t n, uint8_t root[32]) {
  if (!leaves || !root || n == 0) return SG_EINVAL;
  try {
    const auto lv = sg::dns_merkle_levels(leaves, n);
    memcpy(root, lv.back().data(), 32);
    return SG_OK;
  } catch (const std::bad_alloc&) {
    return SG_ENOMEM;
  }
}

int sg_dns_merkle_path(const uint8_t* leaves, size_t n, size_t index, uint8_t* path, size_t cap, size_t* depth) {
  if (!leaves || !depth || n == 0 || index >= n) return SG_EINVAL;
  try {
    const auto p = sg::dns_merkle_path(sg::dns_merkle_levels(leaves, n), index);
    *depth = p.size() / 32;
    if (!path || cap < p.size()) return SG_ESPACE;
    memcpy(path, p.data(), p.size());
    return SG_OK;
  } catch (const std::bad_alloc&) {
    return SG_ENOMEM;
  }
}

int sg_dns_merkle_verify(const uint8_t leaf[32], size_t index, const uint8_t* path, size_t depth,
                         const uint8_t root[32]) {
  if (!leaf || !root || (depth && !path)) return 0;
  return sg::dns_merkle_verify(leaf, index, path, depth, root) ? 1 : 0;
}

void sg_shard_pi_hash(const uint8_t salt[16], uint64_t record_count, const uint8_t merkle_root[32],
                      const uint8_t root_f0[32], const uint8_t fs_binding[32], uint8_t out[32]) {
  sg::shard_pi_hash(salt, record_count, merkle_root, root_f0, fs_binding, out);
}

int sg_prove_inner_shard(sg_ctx* c, const uint8_t* canon, const size_t* offsets, size_t n_records,
                         const uint8_t salt[16], const uint8_t fs_binding[32], int stir, uint8_t* proof, size_t cap,
                         size_t* len, uint8_t pi_hash[32], uint8_t merkle_root[32]) {
  return guarded(c, [&] {
    sg::require(kc::kHashBytes == 32, "prove_inner_shard: swarm-dns binds 32-byte proof roots; it builds with the "
                                      "sha3-256 profile only");
    sg::require(offsets && salt && fs_binding && len && pi_hash && merkle_root && n_records > 0 &&
                    (canon || offsets[n_records] == 0),
                "prove_inner_shard: null argument or no records");
    for (size_t i = 0; i < n_records; ++i)
      sg::require(offsets[i + 1] >= offsets[i], "prove_inner_shard: offsets must not decrease");
    // 1-2. record leaves and the off-chain Merkle root committed in pi_hash
    std::vector<uint8_t> lh(32 * n_records);
    sg::dns_record_leaves(canon, offsets, n_records, salt, lh.data());
    const auto lv = sg::dns_merkle_levels(lh.data(), n_records);
    memcpy(merkle_root, lv.back().data(), 32);
    // 3. every leaf hash as 4 little-endian u64 rollup leaves (pack_hash_to_leaves)
    std::vector<uint64_t> leaves(4 * n_records);
    memcpy(leaves.data(), lh.data(), lh.size());
    std::vector<uint8_t> b =
        sg::prove_hash_rollup_host_leaves(c, leaves.data(), leaves.size(), fs_binding, SG_PHI_PARALLEL_GATE, true,
                                          stir != 0);
    // 4. pi_hash binds salt, count, merkle root, the proof's root_f0 and the FS binding
    sg::shard_pi_hash(salt, n_records, merkle_root, b.data(), fs_binding, pi_hash);
    *len = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_inner_shard: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

int sg_prove_outer_rollup(sg_ctx* c, const uint8_t* pi_hashes, size_t n, const uint8_t pk_hash[32], int stir,
                          uint8_t* proof, size_t cap, size_t* len) {
  return guarded(c, [&] {
    sg::require(kc::kHashBytes == 32, "prove_outer_rollup: swarm-dns binds 32-byte proof roots; it builds with the "
                                      "sha3-256 profile only");
    sg::require(pi_hashes && pk_hash && len && n > 0, "prove_outer_rollup: null argument or no shards");
    std::vector<uint64_t> leaves(4 * n);
    memcpy(leaves.data(), pi_hashes, 32 * n);
    std::vector<uint8_t> b = sg::prove_hash_rollup_host_leaves(c, leaves.data(), leaves.size(), pk_hash,
                                                               SG_PHI_PARALLEL_GATE, true, stir != 0);
    *len = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_outer_rollup: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

int sg_merkle_commit(sg_ctx* c, const uint64_t* cols, size_t n_leaves, size_t width, size_t col_stride,
                     const uint64_t* arities, size_t depth, uint64_t tree_label, uint8_t* root, sg_tree** keep) {
  if (keep) *keep = nullptr;
  return guarded(c, [&] {
    sg::require(cols && root && arities && depth > 0 && n_leaves > 0, "merkle_commit: bad arguments");
    sg::require(width > 0 && col_stride >= n_leaves, "merkle_commit: bad width or column stride");
    std::vector<uint32_t> ar;
    for (size_t i = 0; i < depth; ++i) {
      sg::require(arities[i] >= 2 && arities[i] <= 1024, "merkle_commit: arity out of range");
      ar.push_back((uint32_t)arities[i]);
    }
    In di(cols, (width - 1) * col_stride + n_leaves, c->stream);
    sg_tree* t = new sg_tree;
    try {
      sg::require(sg::tree_plan(&t->t, n_leaves, ar, tree_label), "merkle_commit: arities do not reach the root");
      t->buf.alloc(t->t.total_digests * kc::kDigestLanes, c->stream);
      t->t.d = t->buf.p;
      sg::cuda_check(sg::tree_hash_leaves(t->t, di.d, (uint32_t)width, col_stride, 0, c->stream), "leaves");
      sg::cuda_check(sg::tree_hash_levels(t->t, c->stream), "levels");
      sg::cuda_check(cudaMemcpyAsync(root, t->t.d + kc::kDigestLanes * t->t.off.back(), kc::kHashBytes,
                                     cudaMemcpyDeviceToHost, c->stream),
                     "d2h");
      sg::cuda_check(cudaStreamSynchronize(c->stream), "sync");
    } catch (...) {
      delete t;
      throw;
    }
    if (keep)
      *keep = t;
    else
      delete t;
  });
}

int sg_lde_commit(sg_ctx* c, const uint64_t* trace, size_t w, size_t n_trace, size_t blowup, uint64_t shift,
                  const uint64_t* arities, size_t depth, uint64_t tree_label, uint8_t* root, uint64_t* out,
                  size_t keep_cols, sg_tree** keep) {
  if (keep) *keep = nullptr;
  return guarded(c, [&] {
    sg::require(trace && root && arities && depth > 0, "lde_commit: null argument");
    sg::require(w > 0 && n_trace > 0 && blowup > 0 && keep_cols <= w && (keep_cols == 0 || out),
                "lde_commit: bad shape or kept columns");
    std::vector<uint32_t> ar;
    for (size_t i = 0; i < depth; ++i) {
      sg::require(arities[i] >= 2 && arities[i] <= 1024, "lde_commit: arity out of range");
      ar.push_back((uint32_t)arities[i]);
    }
    const size_t n0 = n_trace * blowup;
    Out dout(out, keep_cols * n0, c->stream);
    sg_tree* t = new sg_tree;
    try {
      sg::require(sg::tree_plan(&t->t, n0, ar, tree_label), "lde_commit: arities do not reach the root");
      t->buf.alloc(t->t.total_digests * kc::kDigestLanes, c->stream);
      t->t.d = t->buf.p;
      sg::lde_commit(c, trace, !sg::is_device_ptr(trace), w, n_trace, blowup, shift, t->t, dout.d, keep_cols);
      sg::cuda_check(sg::tree_hash_levels(t->t, c->stream), "levels");
      sg::cuda_check(cudaMemcpyAsync(root, t->t.d + kc::kDigestLanes * t->t.off.back(), kc::kHashBytes,
                                     cudaMemcpyDeviceToHost, c->stream),
                     "d2h");
      dout.finish();
      sg::cuda_check(cudaStreamSynchronize(c->stream), "sync");
    } catch (...) {
      delete t;
      throw;
    }
    if (keep)
      *keep = t;
    else
      delete t;
  });
}

int sg_merkle_open(sg_ctx* c, const sg_tree* tree, size_t index, uint8_t* out, size_t cap, size_t* len) {
  return guarded(c, [&] {
    sg::require(tree && len, "merkle_open: null tree or length");
    sg::require(index < tree->t.len[0], "merkle_open: index out of range");
    std::vector<uint64_t> idx;
    sg::opening_indices(tree->t, index, &idx);
    sg::DBuf di(idx.size(), c->stream), dout(kc::kDigestLanes * idx.size(), c->stream);
    sg::cuda_check(cudaMemcpyAsync(di.p, idx.data(), idx.size() * 8, cudaMemcpyHostToDevice, c->stream), "h2d");
    sg::cuda_check(sg::gather_digests(tree->t.d, di.p, idx.size(), dout.p, c->stream), "gather");
    std::vector<uint64_t> got(kc::kDigestLanes * idx.size());
    sg::cuda_check(cudaMemcpyAsync(got.data(), dout.p, got.size() * 8, cudaMemcpyDeviceToHost, c->stream), "d2h");
    sg::cuda_check(cudaStreamSynchronize(c->stream), "sync");
    sg::ByteWriter w;
    size_t pos = 0;
    auto dig = [&]() {
      sg::Digest d;
      memcpy(d.data(), got.data() + pos, kc::kHashBytes);
      pos += kc::kDigestLanes;
      return d;
    };
    sg::Opening o;
    o.index = index;
    o.leaf = dig();
    for (size_t l = 0; l + 1 < tree->t.len.size(); ++l) {
      std::vector<sg::Digest> sib(tree->t.arity[l] - 1);
      for (auto& d : sib) d = dig();
      o.path.push_back(std::move(sib));
    }
    w.opening(o);
    *len = w.b.size();
    if (w.b.size() > cap || !out) throw sg::SgError{SG_ESPACE, "merkle_open: output buffer too small"};
    memcpy(out, w.b.data(), w.b.size());
  });
}

void sg_merkle_free(sg_tree* t) { delete t; }

void sg_build_params(size_t n0, const uint8_t* pi32, int stir, sg_fri_params* out) {
  if (!out) return;
  memset(out, 0, sizeof *out);
  unsigned lg = 0;
  while ((size_t(1) << lg) < n0) ++lg;
  if (stir) {
    for (unsigned i = 0; i < lg / 3; ++i) out->schedule[out->schedule_len++] = 8;
    if (lg % 3) out->schedule[out->schedule_len++] = 1ull << (lg % 3);
  } else {
    for (unsigned i = 0; i < lg && i < SG_MAX_SCHEDULE; ++i) out->schedule[out->schedule_len++] = 2;
  }
  out->r = out->s0 = 54;
  out->seed_z = 0xDEEFBAADull;
  out->coeff_commit_final = 1;
  out->d_final = 1;
  out->stir = stir ? 1 : 0;
  if (pi32) {
    out->has_pi = 1;
    memcpy(out->pi_hash, pi32, 32);
  }
}

int sg_stir_prove(sg_ctx* c, const uint64_t* f0, size_t n0, const sg_fri_params* params, uint8_t* proof,
                  size_t cap, size_t* len) {
  return guarded(c, [&] {
    sg::require(f0 && params && len, "stir_prove: null argument");
    sg::require(n0 > 0 && n0 <= (size_t(1) << sg::kMaxLogN), "stir_prove: bad n0");
    In di(f0, n0, c->stream);
    std::vector<uint8_t> b = sg::stir_prove_device(c, di.d, n0, *params);
    *len = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "stir_prove: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

int sg_stir_prove_group(sg_ctx* c, const uint64_t* f0, size_t n0, size_t n_proofs, const sg_fri_params* params,
                        uint8_t* proofs, size_t cap_per_proof, size_t* lens) {
  return guarded(c, [&] {
    sg::require(f0 && params && lens && proofs && n_proofs > 0 && n_proofs <= 4096,
                "stir_prove_group: null argument or bad count");
    sg::require(n0 > 0 && n0 <= (size_t(1) << sg::kMaxLogN), "stir_prove_group: bad n0");
    In di(f0, n0 * n_proofs, c->stream);
    std::vector<sg_fri_params> ps(params, params + n_proofs);
    const auto out = sg::stir_prove_group(c, di.d, n0, n0, ps);
    bool fits = true;
    for (size_t g = 0; g < n_proofs; ++g) {
      lens[g] = out[g].size();
      if (out[g].size() > cap_per_proof) fits = false;
    }
    if (!fits) throw sg::SgError{SG_ESPACE, "stir_prove_group: proof buffer too small"};
    for (size_t g = 0; g < n_proofs; ++g) memcpy(proofs + g * cap_per_proof, out[g].data(), out[g].size());
  });
}

int sg_stir_verify(const uint8_t* proof, size_t len, const sg_fri_params* params) {
  if (!proof || !params) return 0;
  try {
    return sg::stir_verify(sg::decode_proof(proof, len), *params) ? 1 : 0;
  } catch (...) {
    return 0;
  }
}

int sg_prove_hash_rollup(sg_ctx* c, const uint64_t* leaves, size_t n_leaves, const uint8_t pi[32], int phi_mode,
                         uint8_t* proof, size_t cap, size_t* len) {
  return guarded(c, [&] {
    sg::require(len && (leaves || n_leaves == 0), "prove_hash_rollup: null argument");
    std::vector<uint64_t> lv(n_leaves);
    if (n_leaves) {
      if (sg::is_device_ptr(leaves)) {
        sg::cuda_check(cudaMemcpy(lv.data(), leaves, n_leaves * 8, cudaMemcpyDeviceToHost), "d2h");
      } else {
        memcpy(lv.data(), leaves, n_leaves * 8);
      }
    }
    std::vector<uint8_t> b = sg::prove_hash_rollup_host_leaves(c, lv.data(), n_leaves, pi, phi_mode, true);
    *len = b.size();
    if (b.size() > cap || !proof) throw sg::SgError{SG_ESPACE, "prove_hash_rollup: proof buffer too small"};
    memcpy(proof, b.data(), b.size());
  });
}

}  // extern "C"
