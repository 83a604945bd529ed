// ed25519_prover.cu — the Ed25519 verify AIR proof pipeline: witness on the host
// (words and cell codes), trace expanded on the device, LDE x blowup, Phi by the
// gated block kernel plus the SHA-512 kernel for the hash rows, the quotient by
// X^n_trace - 1, and the STIR proof (prove_zsk_ksk_binding_v2,
// swarm-dns/src/prover.rs:856-951).
#include <algorithm>
#include <cstring>

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

// The program's Phi plan and pairs on the device, with lambda_j = j + 1 for the
// SHA-512 block (the first 1526 constraints).
struct PhiDev {
  EdPhiPlan plan;
  DBuf blocks, pairs, cls_list, chunk_rng, cls_chunk, row_class, sha_lam;
  PhiDev(const ed25519::Witness& w, cudaStream_t s) {
    plan = ed25519_phi_plan(w.prog, w.L.height, 2048);
    blocks = upload(plan.blocks, s);
    pairs = upload(w.prog.pairs, s);
    cls_list = upload(plan.cls_list, s);
    chunk_rng = upload(plan.chunk_rng, s);
    cls_chunk = upload(plan.cls_chunk, s);
    row_class = upload(plan.row_class, s);
    std::vector<uint64_t> lam(ed25519::SHA_K);
    for (uint32_t j = 0; j < ed25519::SHA_K; ++j) lam[j] = j + 1;
    sha_lam = upload(lam, s);
  }
  EdPhi args(const uint64_t* lde, uint64_t n, uint64_t blowup, uint64_t n_trace, uint64_t coset_len,
             uint64_t out_stride, uint64_t out_off, const uint64_t* phi_sha, uint64_t sha_rows) const {
    return EdPhi{lde,
                 n,
                 blowup,
                 n_trace,
                 coset_len,
                 out_stride,
                 out_off,
                 (const EdBlock*)blocks.p,
                 pairs.p,
                 (const uint32_t*)cls_list.p,
                 (const uint32_t*)chunk_rng.p,
                 (const uint32_t*)cls_chunk.p,
                 (const uint8_t*)row_class.p,
                 phi_sha,
                 sha_rows,
                 plan.max_chunks};
  }
};

}  // namespace

void ed25519_trace_device(sg_ctx* c, const ed25519::Witness& w, uint64_t* d_trace) {
  const ed25519::Layout& L = w.L;
  cudaStream_t s = c->stream;
  DBuf codes = upload(w.codes, s), phase = upload(w.row_phase, s), off = upload(w.row_off, s);
  DBuf words = upload(w.words, s), globals = upload(w.globals, s), sha = upload(w.sha, s);
  EdExpand d{(const uint32_t*)codes.p, (const uint8_t*)phase.p, (const uint32_t*)off.p, words.p, globals.p, L.width,
             L.height};
  cuda_check(ed25519_expand(d, d_trace, s), "ed25519 trace expand");
  cuda_check(sha512_expand_strided((const sha512::BlockWitness*)sha.p, L.n_blocks, L.k_hash, L.height, d_trace, s),
             "ed25519 sha512 rows");
}

void ed25519_lde_device(sg_ctx* c, const ed25519::Witness& w, const uint64_t* d_trace, uint64_t blowup,
                        uint64_t* d_lde) {
  const ed25519::Layout& L = w.L;
  const ed25519::LdePlan plan = ed25519::make_lde_plan(w);
  if (!plan.ok) {
    lde_device(c, d_trace, L.width, L.height, blowup, 1, d_lde);
    return;
  }
  cudaStream_t s = c->stream;
  lde_device(c, d_trace, plan.dense, L.height, blowup, 1, d_lde);
  std::vector<uint32_t> ar, tasks, nz_rows;
  for (const auto& g : plan.groups) {
    const uint32_t off = (uint32_t)nz_rows.size();
    nz_rows.insert(nz_rows.end(), g.nz.begin(), g.nz.end());
    for (uint32_t a : g.read) {
      const uint32_t lb = (uint32_t)(ar.size() / 2);
      for (uint32_t r : g.nz) ar.push_back(a), ar.push_back(r);
      for (uint32_t col : g.cols) tasks.insert(tasks.end(), {col, a, lb, off, (uint32_t)g.nz.size()});
    }
  }
  DBuf d_ar = upload(ar, s), d_tasks = upload(tasks, s), d_nz = upload(nz_rows, s);
  DBuf d_const = upload(plan.const_cols, s), d_lval(std::max<uint64_t>(1, ar.size() / 2 * blowup), s);
  EdLdeFill f{(const uint32_t*)d_ar.p,    (uint32_t)(ar.size() / 2), (const uint32_t*)d_tasks.p,
              (uint32_t)(tasks.size() / 5), (const uint32_t*)d_nz.p, (const uint32_t*)d_const.p,
              (uint32_t)plan.const_cols.size()};
  cuda_check(ed25519_lde_fill(f, d_trace, L.height, blowup, d_lval.p, d_lde, s), "ed25519 sparse LDE");
}

void ed25519_merge_device(sg_ctx* c, const ed25519::Witness& w, const uint64_t* d_lde, uint64_t blowup,
                          uint64_t* d_c) {
  const ed25519::Layout& L = w.L;
  const uint64_t n_trace = L.height, n = n_trace * blowup;
  const unsigned ln = lg2(n);
  require((1ull << ln) == n && ln <= kMaxLogN, "ed25519 merge: bad sizes");
  cudaStream_t s = c->stream;
  PhiDev pd(w, s);
  const uint64_t sha_rows = L.k_hash - 1;
  DBuf part((uint64_t)pd.plan.max_chunks * n, s), phi(n, s), phi_sha(sha_rows * blowup, s);
  DBuf scratch(ntt_scratch_elems(1, ln), s);
  cuda_check(sha512_phi_points_ex(d_lde, n, n, sha_rows * blowup, blowup, blowup, L.n_blocks, pd.sha_lam.p, phi_sha.p,
                                  1, 0, s),
             "ed25519 sha512 phi");
  cuda_check(ed25519_phi(pd.args(d_lde, n, blowup, n_trace, 0, 1, 0, phi_sha.p, sha_rows), part.p, phi.p, s),
             "ed25519 phi");
  cuda_check(ntt_batch(c->tw, phi.p, phi.p, 1, n, n, (int)ln, true, n, scratch.p, s), "intt");
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  cuda_check(ntt_batch(c->tw, d_c, d_c, 1, n, n, (int)ln, false, n - n_trace, scratch.p, s), "ntt");
}

// LDE point r + blowup a lies on coset r, whose values are NTT_{n_trace}(c_k w_n^{r k})
// of the trace coefficients; the next row of that point is point a + 1 of the same
// coset. Cosets go kCosetGroup at a time, each group's Phi in one launch.
void ed25519_merge_cosets(sg_ctx* c, const ed25519::Witness& w, const uint64_t* d_trace, uint64_t blowup,
                          uint64_t* d_c) {
  constexpr uint64_t kCosetGroup = 8;
  const ed25519::Layout& L = w.L;
  const uint64_t n_trace = L.height, n = n_trace * blowup, W = L.width, G = std::min<uint64_t>(kCosetGroup, blowup);
  const unsigned ln = lg2(n), lt = lg2(n_trace);
  require((1ull << ln) == n && ln <= kMaxLogN, "ed25519 merge: bad sizes");
  cudaStream_t s = c->stream;
  PhiDev pd(w, s);
  const uint64_t sha_rows = L.k_hash - 1;
  DBuf part((uint64_t)pd.plan.max_chunks * G * n_trace, s), phi(n, s), coef(W * n_trace, s), ev(W * G * n_trace, s);
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
    cuda_check(sha512_phi_cosets(ev.p, G, n_trace, sha_rows, L.n_blocks, pd.sha_lam.p, phi_sha.p, s),
               "ed25519 sha512 phi");
    cuda_check(ed25519_phi(pd.args(ev.p, G * n_trace, blowup, n_trace, n_trace, blowup, r0, phi_sha.p, sha_rows),
                           part.p, phi.p, s),
               "ed25519 coset phi");
  }
  cuda_check(ntt_batch(c->tw, phi.p, phi.p, 1, n, n, (int)ln, true, n, scratch.p, s), "intt");
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  cuda_check(ntt_batch(c->tw, d_c, d_c, 1, n, n, (int)ln, false, n - n_trace, scratch.p, s), "ntt");
}

CEval ed25519_ceval(sg_ctx* c, const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, uint64_t len,
                    const uint8_t fs_binding[32], uint32_t k_scalar, uint64_t blowup) {
  check_blowup(blowup);
  ed25519::Witness w;
  ed25519::build_witness(pub, sig, msg, len, k_scalar, &w);
  const uint64_t n0 = (uint64_t)w.L.height * blowup, W = w.L.width;
  cudaStream_t s = c->stream;
  DBuf d_c(n0, s);
  {
    DBuf d_trace(W * w.L.height, s);
    ed25519_trace_device(c, w, d_trace.p);
    // The materialised path transforms only the dense columns (ed25519_lde_device) and
    // is the faster one; streaming by cosets is for callers that cannot hold the LDE.
    const bool cosets = c->wide_merge == SG_WIDE_MERGE_COSETS;
    if (cosets) {
      ed25519_merge_cosets(c, w, d_trace.p, blowup, d_c.p);
    } else {
      DBuf d_lde(W * n0, s);
      ed25519_lde_device(c, w, d_trace.p, blowup, d_lde.p);
      d_trace = DBuf();
      ed25519_merge_device(c, w, d_lde.p, blowup, d_c.p);
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
