// p256_prover.cu — the P-256 ECDSA double-chain proof pipeline: witnesses on the
// host, trace expanded on the device, LDE x32, Phi by the gadget kernel, the
// quotient by X^n_trace - 1, and the STIR proof (prove_ecdsa_record_v1.rs:97-240).
#include <cstring>
#include <mutex>

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

// The layout's device tables (gadget table, cell codes, lambda bases, merge
// chunks, tail bases, b), uploaded once per device and kept for the process.
struct P256Tables {
  const p256::Gadget* table = nullptr;
  const uint32_t *code = nullptr, *lam = nullptr, *chunk = nullptr, *tail = nullptr, *b = nullptr;
  uint32_t n_chunks = 0;
};

template <class T>
const T* upload_const(const T* h, size_t n) {
  void* d = nullptr;
  cuda_check(cudaMalloc(&d, n * sizeof(T)), "p256 tables");
  cuda_check(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice), "p256 tables");
  return (const T*)d;
}

const P256Tables& p256_tables() {
  static std::mutex mu;
  static P256Tables per_dev[64];
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "device");
  require(dev >= 0 && dev < 64, "p256: device index");
  std::lock_guard<std::mutex> g(mu);
  P256Tables& t = per_dev[dev];
  if (!t.table) {
    const p256::Layout& L = p256::layout();
    const std::vector<uint32_t> chunk = p256_chunks(2600);
    t.code = upload_const(L.cell_code.data(), L.cell_code.size());
    t.lam = upload_const(L.lam_base.data(), L.lam_base.size());
    t.chunk = upload_const(chunk.data(), chunk.size());
    t.tail = upload_const(L.tail, 18);
    t.b = upload_const(L.b_limbs, p256::NL);
    t.n_chunks = (uint32_t)chunk.size() - 1;
    t.table = upload_const(L.table.data(), L.table.size());
  }
  return t;
}

}  // namespace

void p256_trace_device(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                       const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, uint64_t k,
                       uint64_t* d_trace) {
  require(k >= 2 && (k & (k - 1)) == 0 && k <= (1u << 16), "p256: rows must be a power of 2 in [2, 65536]");
  const p256::Layout& L = p256::layout();
  const P256Tables& T = p256_tables();
  const uint64_t NG = L.table.size();
  // witnesses straight into pinned staging, so the copy is one fast DMA
  const size_t rows_bytes = k * sizeof(p256::RowW), gw_bytes = k * NG * sizeof(p256::GadgetW);
  const size_t rp_bytes = 6 * p256::NL * sizeof(uint32_t);
  uint8_t* pin = (uint8_t*)pinned_host(c, rows_bytes + gw_bytes + rp_bytes);
  p256::RowW* rows = (p256::RowW*)pin;
  p256::GadgetW* gw = (p256::GadgetW*)(pin + rows_bytes);
  auto rproj = (uint32_t(*)[p256::NL])(pin + rows_bytes + gw_bytes);
  p256::chain_witness(ax, ay, a_bits, bx, by, b_bits, k, rows, gw, rproj);
  cudaStream_t s = c->stream;
  DBuf d_wit((rows_bytes + gw_bytes + rp_bytes + 7) / 8, s);
  cuda_check(cudaMemcpyAsync(d_wit.p, pin, rows_bytes + gw_bytes + rp_bytes, cudaMemcpyHostToDevice, s), "h2d");
  const uint8_t* dw = (const uint8_t*)d_wit.p;
  P256Dev d{T.table, T.code, (const p256::RowW*)dw, (const p256::GadgetW*)(dw + rows_bytes),
            (const uint32_t*)(dw + rows_bytes + gw_bytes), T.b, L.width, (uint32_t)NG};
  cuda_check(p256_expand(d, k, d_trace, s), "p256 trace expand");
  cuda_check(cudaStreamSynchronize(s), "sync");  // the staging buffer is reused by the next proof
}

void p256_merge_device(sg_ctx* c, const uint64_t* d_lde, uint64_t n_trace, uint64_t blowup, uint64_t* d_c) {
  const p256::Layout& L = p256::layout();
  const P256Tables& T = p256_tables();
  const uint64_t n = n_trace * blowup;
  const unsigned ln = lg2(n);
  require((1ull << ln) == n && ln <= kMaxLogN && n_trace >= 2, "p256 merge: bad sizes");
  cudaStream_t s = c->stream;
  DBuf part((uint64_t)T.n_chunks * n, s), phi(n, s), scratch(ntt_scratch_elems(1, ln), s);
  P256Phi a{d_lde, n, blowup, n_trace, 0, 1, 0, T.table, T.lam, T.chunk, T.tail, (uint32_t)L.table.size(),
            L.n_constraints - p256::TAIL_CONSTRAINTS};
  cuda_check(p256_phi(a, T.n_chunks, part.p, phi.p, s), "p256 phi");
  cuda_check(ntt_batch(c->tw, phi.p, phi.p, 1, n, n, (int)ln, true, n, scratch.p, s), "intt");
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  cuda_check(ntt_batch(c->tw, d_c, d_c, 1, n, n, (int)ln, false, n - n_trace, scratch.p, s), "ntt");
}

// The same merge without materialising the LDE (the reference's streaming merge,
// deep_ali_merge_ecdsa_double_multirow_streaming, lib.rs:1421-1681, which also
// never holds the whole LDE): LDE point r + blowup a lies on coset r, whose
// values are NTT_{n_trace}(c_k w_n^{r k}) of the trace coefficients c, and the
// next row of that point is point a + 1 of the same coset. Each coset is
// produced, its Phi values are written to Phi[r + blowup a], and it is dropped.
// Cosets go kCosetGroup at a time (their evaluations one after another), so each
// Phi launch covers kCosetGroup x n_trace points: one coset alone (256 points for
// K = 256) gives the constraint kernel too few CTAs to fill the GPU. The device
// holds the trace, its coefficients and one group (2 x 310 MB + 2.5 GB for K = 256)
// instead of the 9.9 GB LDE.
void p256_merge_cosets(sg_ctx* c, const uint64_t* d_trace, uint64_t n_trace, uint64_t blowup, uint64_t* d_c) {
  constexpr uint64_t kCosetGroup = 8;
  const p256::Layout& L = p256::layout();
  const P256Tables& T = p256_tables();
  const uint64_t n = n_trace * blowup, W = L.width, G = std::min<uint64_t>(kCosetGroup, blowup);
  const unsigned ln = lg2(n), lt = lg2(n_trace);
  require((1ull << ln) == n && (1ull << lt) == n_trace && ln <= kMaxLogN && n_trace >= 2, "p256 merge: bad sizes");
  cudaStream_t s = c->stream;
  DBuf part((uint64_t)T.n_chunks * G * n_trace, s), phi(n, s), coef(W * n_trace, s), ev(W * G * n_trace, s);
  DBuf scratch(std::max(ntt_scratch_elems((uint32_t)W, (int)lt), ntt_scratch_elems(1, (int)ln)), s);
  DBuf twist_tab(n_trace, s);
  cuda_check(ntt_batch(c->tw, d_trace, coef.p, (uint32_t)W, n_trace, n_trace, (int)lt, true, n_trace, scratch.p, s),
             "p256 trace intt");
  for (uint64_t r0 = 0; r0 < blowup; r0 += G) {
    // column col of coset r0 + g at ev[col * G n_trace + g n_trace]
    for (uint64_t g = 0; g < G; ++g) {
      const uint64_t r = r0 + g;
      PowSpec twist;
      if (r > 0) {
        cuda_check(pow_table_device(c->tw, r, (int)ln, n_trace, twist_tab.p, s), "twist table");
        twist.tab = twist_tab.p;
      }
      cuda_check(ntt_batch(c->tw, coef.p, ev.p + g * n_trace, (uint32_t)W, n_trace, G * n_trace, (int)lt, false,
                           n_trace, scratch.p, s, r > 0 ? &twist : nullptr),
                 "p256 coset ntt");
    }
    P256Phi a{ev.p, G * n_trace, blowup, n_trace, n_trace, blowup, r0, T.table, T.lam, T.chunk, T.tail,
              (uint32_t)L.table.size(), L.n_constraints - p256::TAIL_CONSTRAINTS};
    cuda_check(p256_phi(a, T.n_chunks, part.p, phi.p, s), "p256 coset phi");
  }
  cuda_check(ntt_batch(c->tw, phi.p, phi.p, 1, n, n, (int)ln, true, n, scratch.p, s), "intt");
  cuda_check(quotient_zh(phi.p, n, n_trace, d_c, s), "quotient");
  cuda_check(ntt_batch(c->tw, d_c, d_c, 1, n, n, (int)ln, false, n - n_trace, scratch.p, s), "ntt");
}

CEval p256_chains_ceval(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                        const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, uint64_t k,
                        const uint8_t pi[32], uint64_t blowup) {
  const p256::Layout& L = p256::layout();
  require(blowup >= 2 && blowup <= 1024 && !(blowup & (blowup - 1)), "prove: blowup must be a power of 2 in [2, 1024]");
  const uint64_t n0 = k * blowup, W = L.width;
  cudaStream_t s = c->stream;
  DBuf d_c(n0, s);
  {
    DBuf d_trace(W * k, s);
    p256_trace_device(c, ax, ay, a_bits, bx, by, b_bits, k, d_trace.p);
    const bool cosets = c->wide_merge == SG_WIDE_MERGE_COSETS ||
                        (c->wide_merge == SG_WIDE_MERGE_AUTO && W * n0 * 8 > (2ull << 30));
    if (cosets) {
      p256_merge_cosets(c, d_trace.p, k, blowup, d_c.p);
    } else {
      DBuf d_lde(W * n0, s);
      lde_device(c, d_trace.p, W, k, blowup, 1, d_lde.p);
      d_trace = DBuf();
      p256_merge_device(c, d_lde.p, k, blowup, d_c.p);
    }
  }
  CEval r;
  r.d_c = std::move(d_c);
  r.n0 = n0;
  sg_build_params(n0, pi, 1, &r.params);
  return r;
}

std::vector<uint8_t> prove_p256_chains(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                                       const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, uint64_t k,
                                       const uint8_t pi[32], bool self_verify, uint64_t blowup) {
  return prove_from_ceval(c, p256_chains_ceval(c, ax, ay, a_bits, bx, by, b_bits, k, pi, blowup), self_verify);
}

CEval p256_ecdsa_ceval(sg_ctx* c, const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32],
                       const uint8_t sgn[32], const uint8_t digest[32], const uint8_t pi[32], uint64_t blowup) {
  uint8_t u1[256], u2[256];
  p256::u_bits(digest, r, sgn, u1, u2);
  return p256_chains_ceval(c, p256::GX, p256::GY, u1, qx, qy, u2, p256::K_ECDSA, pi, blowup);
}

std::vector<uint8_t> prove_p256_ecdsa(sg_ctx* c, const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32],
                                      const uint8_t sgn[32], const uint8_t digest[32], const uint8_t pi[32],
                                      bool self_verify, uint64_t blowup) {
  uint8_t u1[256], u2[256];
  p256::u_bits(digest, r, sgn, u1, u2);
  return prove_p256_chains(c, p256::GX, p256::GY, u1, qx, qy, u2, p256::K_ECDSA, pi, self_verify, blowup);
}

}  // namespace sg
