// p256_prover.hpp — P-256 ECDSA double-chain pipeline entry points used by the C ABI.
#pragma once
#include <cstdint>
#include <vector>

#include "context.hpp"
#include "prover.hpp"

namespace sg {

// (width x k) trace of two chains (chain A from (ax, ay, 1) with a_bits, chain B
// from (bx, by, 1) with b_bits; bits are bytes 0/1) into device memory.
void p256_trace_device(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                       const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, uint64_t k,
                       uint64_t* d_trace);
// Phi + quotient on a materialised (width x n_trace*blowup) LDE.
void p256_merge_device(sg_ctx* c, const uint64_t* d_lde, uint64_t n_trace, uint64_t blowup, uint64_t* d_c);
// trace -> LDE x32 -> merge -> STIR with build_params(k * 32, pi).
std::vector<uint8_t> prove_p256_chains(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                                       const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, uint64_t k,
                                       const uint8_t pi[32], bool self_verify, uint64_t blowup = 32);
// c_eval of the same proofs (everything before the STIR phase).
CEval p256_chains_ceval(sg_ctx* c, const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits,
                        const uint8_t bx[32], const uint8_t by[32], const uint8_t* b_bits, uint64_t k,
                        const uint8_t pi[32], uint64_t blowup = 32);
CEval p256_ecdsa_ceval(sg_ctx* c, const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32],
                       const uint8_t s[32], const uint8_t digest[32], const uint8_t pi[32], uint64_t blowup = 32);
// prove_ecdsa_record_v1.rs:97-240: chain A = u1 bits from G, chain B = u2 bits from Q, K = 256.
std::vector<uint8_t> prove_p256_ecdsa(sg_ctx* c, const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32],
                                      const uint8_t s[32], const uint8_t digest[32], const uint8_t pi[32],
                                      bool self_verify, uint64_t blowup = 32);

}  // namespace sg
