// ed25519_prover.cu — the Ed25519 verify AIR proof pipeline: witness on the host
// (words and cell codes), trace expanded on the device, LDE x blowup, Phi by the
// gated block kernel plus the SHA-512 kernel for the hash rows, the quotient by
// X^n_trace - 1, and the STIR proof (prove_zsk_ksk_binding_v2,
// swarm-dns/src/prover.rs:856-951).
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

#include "context.hpp"
#include "ed25519_air.cuh"
#include "ed25519_prover.hpp"
#include "merge.cuh"
#include "ntt.cuh"
#include "sha512_air.cuh"

namespace sg {
namespace {

unsigned lg2(uint64_t n) {
  unsigned l = 0;
  while ((1ull << l) < n) ++l;
  return l;
}

template <class T>
DBuf upload(const T* h, size_t n, cudaStream_t s) {
  DBuf d((n * sizeof(T) + 7) / 8, s);
  if (n) cuda_check(cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, s), "ed25519 h2d");
  return d;
}
template <class T>
DBuf upload(const std::vector<T>& v, cudaStream_t s) {
  return upload(v.data(), v.size(), s);
}

// Everything that depends only on a proof's shape (k_scalar and the SHA-512 block
// count): the per-phase cell codes, the row phases and word offsets, the Phi plan
// (row classes and block chunks), the sparse-LDE plan with its Lagrange pairs and
// fill tasks, and lambda_j = j + 1 for the SHA-512 block. The first witness of a
// shape builds it; on each device up to kMaxShapes shapes stay resident for the
// process, and every later witness is compared with the shape before it is used.
struct EdShape {
  std::vector<uint32_t> codes, row_off;
  std::vector<uint8_t> row_phase;
  std::vector<ed25519::Block> blocks;
  std::vector<uint64_t> pair_refs;  // the program's pairs with their constants zeroed
  EdPhiPlan phi;
  ed25519::LdePlan lde;
  std::vector<uint32_t> ar, tasks, nz_rows;  // Lagrange (read row, non-zero row) pairs; 5 words a task
  // device copies
  const uint32_t *d_codes = nullptr, *d_off = nullptr, *d_cls_list = nullptr, *d_chunk_rng = nullptr,
                 *d_cls_chunk = nullptr, *d_ar = nullptr, *d_tasks = nullptr, *d_nz = nullptr, *d_const = nullptr;
  const uint8_t *d_phase = nullptr, *d_row_class = nullptr;
  const EdBlock* d_blocks = nullptr;
  const uint64_t* d_sha_lam = nullptr;
  std::vector<DBuf> own;  // a shape built for one proof owns its tables
};

constexpr int kMaxShapes = 32;

std::vector<uint64_t> pair_refs(const ed25519::Program& p) {
  std::vector<uint64_t> r(p.pairs);
  for (uint64_t& x : r)
    if ((x >> 62) == ed25519::SRC_CONST) x = ed25519::SRC_CONST << 62;
  return r;
}

bool same_shape(const EdShape& sh, const ed25519::Witness& w) {
  const auto& b = w.prog.blocks;
  return w.codes == sh.codes && w.row_phase == sh.row_phase && w.row_off == sh.row_off &&
         b.size() == sh.blocks.size() && !memcmp(b.data(), sh.blocks.data(), b.size() * sizeof(ed25519::Block)) &&
         pair_refs(w.prog) == sh.pair_refs;
}

// A resident table (cudaMalloc, kept for the process) or, for a one-proof shape, a
// stream-ordered buffer the shape owns.
template <class T>
const T* place(EdShape& sh, const std::vector<T>& v, bool resident, cudaStream_t s) {
  if (!resident) {
    sh.own.push_back(upload(v, s));
    return (const T*)sh.own.back().p;
  }
  void* d = nullptr;
  const size_t bytes = v.size() * sizeof(T);
  cuda_check(cudaMalloc(&d, std::max<size_t>(bytes, 16)), "ed25519 shape tables");
  if (bytes) cuda_check(cudaMemcpy(d, v.data(), bytes, cudaMemcpyHostToDevice), "ed25519 shape tables");
  return (const T*)d;
}

std::shared_ptr<EdShape> make_shape(const ed25519::Witness& w, bool resident, cudaStream_t s) {
  auto sh = std::make_shared<EdShape>();
  EdShape& S = *sh;
  S.codes = w.codes;
  S.row_off = w.row_off;
  S.row_phase = w.row_phase;
  S.blocks = w.prog.blocks;
  S.pair_refs = pair_refs(w.prog);
  S.phi = ed25519_phi_plan(w.prog, w.L.height, 1024);
  S.lde = ed25519::make_lde_plan(w);
  for (const auto& g : S.lde.groups) {
    const uint32_t off = (uint32_t)S.nz_rows.size();
    S.nz_rows.insert(S.nz_rows.end(), g.nz.begin(), g.nz.end());
    for (uint32_t a : g.read) {
      const uint32_t lb = (uint32_t)(S.ar.size() / 2);
      for (uint32_t r : g.nz) S.ar.push_back(a), S.ar.push_back(r);
      for (uint32_t col : g.cols) S.tasks.insert(S.tasks.end(), {col, a, lb, off, (uint32_t)g.nz.size()});
    }
  }
  std::vector<uint64_t> lam(ed25519::SHA_K);
  for (uint32_t j = 0; j < ed25519::SHA_K; ++j) lam[j] = j + 1;
  S.d_codes = place(S, S.codes, resident, s);
  S.d_off = place(S, S.row_off, resident, s);
  S.d_phase = place(S, S.row_phase, resident, s);
  S.d_blocks = place(S, S.phi.blocks, resident, s);
  S.d_cls_list = place(S, S.phi.cls_list, resident, s);
  S.d_chunk_rng = place(S, S.phi.chunk_rng, resident, s);
  S.d_cls_chunk = place(S, S.phi.cls_chunk, resident, s);
  S.d_row_class = place(S, S.phi.row_class, resident, s);
  S.d_sha_lam = place(S, lam, resident, s);
  S.d_ar = place(S, S.ar, resident, s);
  S.d_tasks = place(S, S.tasks, resident, s);
  S.d_nz = place(S, S.nz_rows, resident, s);
  S.d_const = place(S, S.lde.const_cols, resident, s);
  return sh;
}

std::shared_ptr<const EdShape> shape_for(sg_ctx* c, const ed25519::Witness& w) {
  static std::mutex mu;
  static std::map<std::tuple<int, uint32_t, uint32_t>, std::shared_ptr<const EdShape>> resident;
  static std::map<int, int> per_device;
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "device");
  const auto key = std::make_tuple(dev, w.L.k, w.L.n_blocks);
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = resident.find(key);
    if (it != resident.end()) {
      if (same_shape(*it->second, w)) return it->second;
    } else if (per_device[dev] < kMaxShapes) {
      ++per_device[dev];
      return resident[key] = make_shape(w, true, c->stream);
    }
  }
  return make_shape(w, false, c->stream);
}

// A proof's own device inputs (its words, globals, SHA-512 block witnesses and the
// program's pairs), copied in one transfer through the context's pinned staging.
struct EdInputs {
  DBuf buf;
  const uint64_t *words = nullptr, *globals = nullptr, *pairs = nullptr;
  const sha512::BlockWitness* sha = nullptr;
};

EdInputs upload_inputs(sg_ctx* c, const ed25519::Witness& w) {
  auto r16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
  const size_t bw = r16(w.words.size() * 8), bg = r16(w.globals.size() * 8), bp = r16(w.prog.pairs.size() * 8),
               bs = r16(w.sha.size() * sizeof(sha512::BlockWitness)), total = bw + bg + bp + bs;
  uint8_t* pin = (uint8_t*)pinned_host(c, total);
  memcpy(pin, w.words.data(), w.words.size() * 8);
  memcpy(pin + bw, w.globals.data(), w.globals.size() * 8);
  memcpy(pin + bw + bg, w.prog.pairs.data(), w.prog.pairs.size() * 8);
  memcpy(pin + bw + bg + bp, w.sha.data(), w.sha.size() * sizeof(sha512::BlockWitness));
  EdInputs in;
  cudaStream_t s = c->stream;
  in.buf.alloc(total / 8, s);
  cuda_check(cudaMemcpyAsync(in.buf.p, pin, total, cudaMemcpyHostToDevice, s), "ed25519 inputs h2d");
  const uint8_t* d = (const uint8_t*)in.buf.p;
  in.words = (const uint64_t*)d;
  in.globals = (const uint64_t*)(d + bw);
  in.pairs = (const uint64_t*)(d + bw + bg);
  in.sha = (const sha512::BlockWitness*)(d + bw + bg + bp);
  cuda_check(cudaStreamSynchronize(s), "sync");  // the staging buffer is reused by the next proof
  return in;
}

EdPhi phi_args(const EdShape& S, const uint64_t* pairs, const uint64_t* lde, uint64_t n, uint64_t blowup,
               uint64_t n_trace, uint64_t coset_len, uint64_t out_stride, uint64_t out_off, const uint64_t* phi_sha,
               uint64_t sha_rows) {
  return EdPhi{lde,          n,        blowup,         n_trace,          coset_len,
               out_stride,   out_off,  S.d_blocks,     pairs,            S.d_cls_list,
               S.d_chunk_rng, S.d_cls_chunk, S.d_row_class, phi_sha,      sha_rows,
               S.phi.max_chunks};
}

void trace_on_device(sg_ctx* c, const ed25519::Witness& w, const EdShape& S, const EdInputs& in, uint64_t* d_trace) {
  const ed25519::Layout& L = w.L;
  cudaStream_t s = c->stream;
  EdExpand d{S.d_codes, S.d_phase, S.d_off, in.words, in.globals, L.width, L.height};
  cuda_check(ed25519_expand(d, d_trace, s), "ed25519 trace expand");
  cuda_check(sha512_expand_strided(in.sha, L.n_blocks, L.k_hash, L.height, d_trace, s), "ed25519 sha512 rows");
}

void lde_on_device(sg_ctx* c, const ed25519::Witness& w, const EdShape& S, const uint64_t* d_trace, uint64_t blowup,
                   uint64_t* d_lde) {
  const ed25519::Layout& L = w.L;
  if (!S.lde.ok) {
    lde_device(c, d_trace, L.width, L.height, blowup, 1, d_lde);
    return;
  }
  cudaStream_t s = c->stream;
  lde_device(c, d_trace, S.lde.dense, L.height, blowup, 1, d_lde);
  const uint32_t n_pairs = (uint32_t)(S.ar.size() / 2);
  DBuf d_lval(std::max<uint64_t>(1, (uint64_t)n_pairs * blowup), s);
  EdLdeFill f{S.d_ar, n_pairs, S.d_tasks, (uint32_t)(S.tasks.size() / 5), S.d_nz, S.d_const,
              (uint32_t)S.lde.const_cols.size()};
  cuda_check(ed25519_lde_fill(f, d_trace, L.height, blowup, d_lval.p, d_lde, s), "ed25519 sparse LDE");
}

void merge_on_device(sg_ctx* c, const ed25519::Witness& w, const EdShape& S, const uint64_t* pairs,
                     const uint64_t* d_lde, uint64_t blowup, uint64_t* d_c) {
  const ed25519::Layout& L = w.L;
  const uint64_t n_trace = L.height, n = n_trace * blowup;
  const unsigned ln = lg2(n);
  require((1ull << ln) == n && ln <= kMaxLogN, "ed25519 merge: bad sizes");
  cudaStream_t s = c->stream;
  const uint64_t sha_rows = L.k_hash - 1;
  DBuf part((uint64_t)S.phi.max_chunks * n, s), phi(n, s), phi_sha(sha_rows * blowup, s);
  DBuf scratch(ntt_scratch_elems(1, ln), s);
  // The SHA-512 block's Phi on the hash rows (a few dozen CTAs, latency-bound) runs on
  // the context's second stream beside the block kernel; the sum waits for both.
  if (!c->copy_stream) cuda_check(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking), "side stream");
  cudaEvent_t fork = nullptr, join = nullptr;
  cuda_check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
  cuda_check(cudaEventCreateWithFlags(&join, cudaEventDisableTiming), "event");
  try {
    cuda_check(cudaEventRecord(fork, s), "event");
    cuda_check(cudaStreamWaitEvent(c->copy_stream, fork, 0), "wait");
    cuda_check(sha512_phi_points_ex(d_lde, n, n, sha_rows * blowup, blowup, blowup, L.n_blocks, S.d_sha_lam,
                                    phi_sha.p, 1, 0, c->copy_stream),
               "ed25519 sha512 phi");
    cuda_check(cudaEventRecord(join, c->copy_stream), "event");
    const EdPhi a = phi_args(S, pairs, d_lde, n, blowup, n_trace, 0, 1, 0, phi_sha.p, sha_rows);
    cuda_check(ed25519_phi_blocks(a, part.p, s), "ed25519 phi");
    cuda_check(cudaStreamWaitEvent(s, join, 0), "wait");
    cuda_check(ed25519_phi_add(a, part.p, phi.p, s), "ed25519 phi sum");
  } catch (...) {
    cudaStreamWaitEvent(s, join, 0);
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
    throw;
  }
  cudaEventDestroy(fork);
  cudaEventDestroy(join);
  cuda_check(ntt_batch(c->tw, phi.p, phi.p, 1, n, n, (int)ln, true, n, scratch.p, s), "intt");
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  cuda_check(ntt_batch(c->tw, d_c, d_c, 1, n, n, (int)ln, false, n - n_trace, scratch.p, s), "ntt");
}

// LDE point r + blowup a lies on coset r, whose values are NTT_{n_trace}(c_k w_n^{r k})
// of the trace coefficients; the next row of that point is point a + 1 of the same
// coset. Cosets go kCosetGroup at a time, each group's Phi in one launch.
void merge_cosets_on_device(sg_ctx* c, const ed25519::Witness& w, const EdShape& S, const uint64_t* pairs,
                            const uint64_t* d_trace, uint64_t blowup, uint64_t* d_c) {
  constexpr uint64_t kCosetGroup = 8;
  const ed25519::Layout& L = w.L;
  const uint64_t n_trace = L.height, n = n_trace * blowup, W = L.width, G = std::min<uint64_t>(kCosetGroup, blowup);
  const unsigned ln = lg2(n), lt = lg2(n_trace);
  require((1ull << ln) == n && ln <= kMaxLogN, "ed25519 merge: bad sizes");
  cudaStream_t s = c->stream;
  const uint64_t sha_rows = L.k_hash - 1;
  DBuf part((uint64_t)S.phi.max_chunks * G * n_trace, s), phi(n, s), coef(W * n_trace, s), ev(W * G * n_trace, s);
  DBuf phi_sha(G * n_trace, s);
  DBuf scratch(std::max(ntt_scratch_elems((uint32_t)W, (int)lt), ntt_scratch_elems(1, (int)ln)), s);
  DBuf twist_tab(n_trace, s);
  cuda_check(ntt_batch(c->tw, d_trace, coef.p, (uint32_t)W, n_trace, n_trace, (int)lt, true, n_trace, scratch.p, s),
             "ed25519 trace intt");
  for (uint64_t r0 = 0; r0 < blowup; r0 += G) {
    for (uint64_t g = 0; g < G; ++g) {
      const uint64_t r = r0 + g;
      PowSpec twist;
      if (r > 0) {
        cuda_check(pow_table_device(c->tw, r, (int)ln, n_trace, twist_tab.p, s), "twist table");
        twist.tab = twist_tab.p;
      }
      cuda_check(ntt_batch(c->tw, coef.p, ev.p + g * n_trace, (uint32_t)W, n_trace, G * n_trace, (int)lt, false,
                           n_trace, scratch.p, s, r > 0 ? &twist : nullptr),
                 "ed25519 coset ntt");
    }
    cuda_check(sha512_phi_cosets(ev.p, G, n_trace, sha_rows, L.n_blocks, S.d_sha_lam, phi_sha.p, s),
               "ed25519 sha512 phi");
    cuda_check(ed25519_phi(phi_args(S, pairs, ev.p, G * n_trace, blowup, n_trace, n_trace, blowup, r0, phi_sha.p,
                                    sha_rows),
                           part.p, phi.p, s),
               "ed25519 coset phi");
  }
  cuda_check(ntt_batch(c->tw, phi.p, phi.p, 1, n, n, (int)ln, true, n, scratch.p, s), "intt");
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  cuda_check(ntt_batch(c->tw, d_c, d_c, 1, n, n, (int)ln, false, n - n_trace, scratch.p, s), "ntt");
}

}  // namespace

void ed25519_trace_device(sg_ctx* c, const ed25519::Witness& w, uint64_t* d_trace) {
  const auto S = shape_for(c, w);
  const EdInputs in = upload_inputs(c, w);
  trace_on_device(c, w, *S, in, d_trace);
}

void ed25519_lde_device(sg_ctx* c, const ed25519::Witness& w, const uint64_t* d_trace, uint64_t blowup,
                        uint64_t* d_lde) {
  lde_on_device(c, w, *shape_for(c, w), d_trace, blowup, d_lde);
}

void ed25519_merge_device(sg_ctx* c, const ed25519::Witness& w, const uint64_t* d_lde, uint64_t blowup,
                          uint64_t* d_c) {
  const auto S = shape_for(c, w);
  const EdInputs in = upload_inputs(c, w);
  merge_on_device(c, w, *S, in.pairs, d_lde, blowup, d_c);
}

void ed25519_merge_cosets(sg_ctx* c, const ed25519::Witness& w, const uint64_t* d_trace, uint64_t blowup,
                          uint64_t* d_c) {
  const auto S = shape_for(c, w);
  const EdInputs in = upload_inputs(c, w);
  merge_cosets_on_device(c, w, *S, in.pairs, d_trace, blowup, d_c);
}

CEval ed25519_ceval(sg_ctx* c, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, uint64_t len,
                    const uint8_t fs_binding[32], uint32_t k_scalar, uint64_t blowup) {
  check_blowup(blowup);
  ed25519::Witness w;
  ed25519::build_witness(pub, sig, msg, len, k_scalar, &w);
  const auto S = shape_for(c, w);
  const uint64_t n0 = (uint64_t)w.L.height * blowup, W = w.L.width;
  cudaStream_t s = c->stream;
  const EdInputs in = upload_inputs(c, w);
  DBuf d_c(n0, s);
  {
    DBuf d_trace(W * w.L.height, s);
    trace_on_device(c, w, *S, in, d_trace.p);
    // The materialised path transforms only the dense columns (lde_on_device) and is
    // the faster one; streaming by cosets is for callers that cannot hold the LDE.
    if (c->wide_merge == SG_WIDE_MERGE_COSETS) {
      merge_cosets_on_device(c, w, *S, in.pairs, d_trace.p, blowup, d_c.p);
    } else {
      DBuf d_lde(W * n0, s);
      lde_on_device(c, w, *S, d_trace.p, blowup, d_lde.p);
      d_trace = DBuf();
      merge_on_device(c, w, *S, in.pairs, d_lde.p, blowup, d_c.p);
    }
  }
  CEval r;
  r.d_c = std::move(d_c);
  r.n0 = n0;
  sg_build_params(n0, fs_binding, 1, &r.params);
  return r;
}

std::vector<uint8_t> prove_ed25519(sg_ctx* c, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg,
                                   uint64_t len, const uint8_t fs_binding[32], uint32_t k_scalar, bool self_verify,
                                   uint64_t blowup) {
  return prove_from_ceval(c, ed25519_ceval(c, pub, sig, msg, len, fs_binding, k_scalar, blowup), self_verify);
}

}  // namespace sg
