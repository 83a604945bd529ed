// p256_prover.cu — the P-256 ECDSA double-chain proof pipeline: witnesses on the
// host, trace expanded on the device, LDE x32, Phi by the gadget kernel, the
// quotient by X^n_trace - 1, and the STIR proof (prove_ecdsa_record_v1.rs:97-240).
#include <cstring>

#include "context.hpp"
#include "merge.cuh"
#include "ntt.cuh"
#include "p256_air.cuh"
#include "p256_prover.hpp"
#include "prover.hpp"
#include "verifier.hpp"

namespace sg {
namespace {

unsigned lg2(uint64_t n) {
  unsigned l = 0;
  while ((1ull << l) < n) ++l;
  return l;
}

template <class T>
void h2d(DBuf* d, const std::vector<T>& v, cudaStream_t s) {
  d->alloc((v.size() * sizeof(T) + 7) / 8, s);
  cuda_check(cudaMemcpyAsync(d->p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), "h2d");
}

}  // namespace

void p256_trace_device(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                       const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, uint64_t k,
                       uint64_t* d_trace) {
  require(k >= 2 && (k & (k - 1)) == 0 && k <= (1u << 16), "p256: rows must be a power of 2 in [2, 65536]");
  const p256::Layout& L = p256::layout();
  std::vector<p256::RowW> rows;
  std::vector<p256::GadgetW> gw;
  uint32_t rproj[6][p256::NL];
  p256::chain_witness(ax, ay, a_bits, bx, by, b_bits, k, &rows, &gw, rproj);
  cudaStream_t s = c->stream;
  DBuf d_table, d_code, d_rows, d_gw, d_rp, d_b;
  h2d(&d_table, L.table, s);
  h2d(&d_code, L.cell_code, s);
  h2d(&d_rows, rows, s);
  h2d(&d_gw, gw, s);
  h2d(&d_rp, std::vector<uint32_t>(&rproj[0][0], &rproj[0][0] + 6 * p256::NL), s);
  h2d(&d_b, std::vector<uint32_t>(L.b_limbs, L.b_limbs + p256::NL), s);
  P256Dev d{(const p256::Gadget*)d_table.p, (const uint32_t*)d_code.p, (const p256::RowW*)d_rows.p,
            (const p256::GadgetW*)d_gw.p, (const uint32_t*)d_rp.p, (const uint32_t*)d_b.p, L.width,
            (uint32_t)L.table.size()};
  cuda_check(p256_expand(d, k, d_trace, s), "p256 trace expand");
  cuda_check(cudaStreamSynchronize(s), "sync");  // host witnesses must outlive their copies
}

void p256_merge_device(sg_ctx* c, const uint64_t* d_lde, uint64_t n_trace, uint64_t blowup, uint64_t* d_c) {
  const p256::Layout& L = p256::layout();
  const uint64_t n = n_trace * blowup;
  const unsigned ln = lg2(n);
  require((1ull << ln) == n && ln <= kMaxLogN && n_trace >= 2, "p256 merge: bad sizes");
  cudaStream_t s = c->stream;
  const std::vector<uint32_t> chunk = p256_chunks(2600);
  const uint32_t n_chunks = (uint32_t)chunk.size() - 1;
  DBuf d_table, d_lam, d_chunk, d_tail;
  h2d(&d_table, L.table, s);
  h2d(&d_lam, L.lam_base, s);
  h2d(&d_chunk, chunk, s);
  h2d(&d_tail, std::vector<uint32_t>(L.tail, L.tail + 18), s);
  DBuf part((uint64_t)n_chunks * n, s), phi(n, s), scratch(ntt_scratch_elems(1, ln), s);
  P256Phi a{d_lde, n, blowup, n_trace, (const p256::Gadget*)d_table.p, (const uint32_t*)d_lam.p,
            (const uint32_t*)d_chunk.p, (const uint32_t*)d_tail.p, (uint32_t)L.table.size(),
            L.n_constraints - p256::TAIL_CONSTRAINTS};
  cuda_check(p256_phi(a, n_chunks, part.p, phi.p, s), "p256 phi");
  cuda_check(ntt_batch(c->tw, phi.p, phi.p, 1, n, n, (int)ln, true, n, scratch.p, s), "intt");
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  cuda_check(ntt_batch(c->tw, d_c, d_c, 1, n, n, (int)ln, false, n - n_trace, scratch.p, s), "ntt");
  cuda_check(cudaStreamSynchronize(s), "sync");  // host tables must outlive their copies
}

std::vector<uint8_t> prove_p256_chains(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                                       const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, uint64_t k,
                                       const uint8_t pi[32], bool self_verify) {
  const p256::Layout& L = p256::layout();
  const uint64_t blowup = p256::BLOWUP, n0 = k * blowup, W = L.width;
  cudaStream_t s = c->stream;
  DBuf d_c(n0, s);
  {
    DBuf d_trace(W * k, s);
    p256_trace_device(c, ax, ay, a_bits, bx, by, b_bits, k, d_trace.p);
    DBuf d_lde(W * n0, s);
    lde_device(c, d_trace.p, W, k, blowup, 1, d_lde.p);
    d_trace = DBuf();
    p256_merge_device(c, d_lde.p, k, blowup, d_c.p);
  }
  sg_fri_params p;
  sg_build_params(n0, pi, 1, &p);
  std::vector<uint8_t> proof = stir_prove_device(c, d_c.p, n0, p);
  if (self_verify && !stir_verify(decode_proof(proof.data(), proof.size()), p))
    throw SgError{SG_EVERIFY, "self-verification of the produced proof failed"};
  return proof;
}

std::vector<uint8_t> prove_p256_ecdsa(sg_ctx* c, const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32],
                                      const uint8_t sgn[32], const uint8_t digest[32], const uint8_t pi[32],
                                      bool self_verify) {
  uint8_t u1[256], u2[256];
  p256::u_bits(digest, r, sgn, u1, u2);
  return prove_p256_chains(c, p256::GX, p256::GY, u1, qx, qy, u2, p256::K_ECDSA, pi, self_verify);
}

}  // namespace sg
