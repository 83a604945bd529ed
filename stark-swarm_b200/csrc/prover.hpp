// prover.hpp — device pipeline entry points used by the C ABI.
#pragma once
#include <cstdint>
#include <vector>

#include "context.hpp"
#include "hash_air.hpp"
#include "merkle.cuh"
#include "protocol.hpp"
#include "rsa2048.hpp"

namespace sg {

// The composition codeword c_eval of a proof (deep_fri_prove's f0, n0 values on
// the device) and its FRI parameters: everything a prover does before the STIR
// phase. A group of them with the same n0 goes through stir_prove_group.
struct CEval {
  DBuf d_c;
  uint64_t n0 = 0;
  sg_fri_params params{};
};
// STIR of c_eval, then (optionally) self-verification; the prove_* entries below
// are their *_ceval functions followed by this.
std::vector<uint8_t> prove_from_ceval(sg_ctx* c, const CEval& ce, bool self_verify);

void lde_device(sg_ctx* c, const uint64_t* d_trace, uint64_t w, uint64_t n_trace, uint64_t blowup, uint64_t shift,
                uint64_t* d_out);
// lde_device from a host trace, its copy pipelined with the transform by column chunks.
void lde_from_host(sg_ctx* c, const uint64_t* h_trace, uint64_t w, uint64_t n_trace, uint64_t blowup, uint64_t shift,
                   uint64_t* d_out);
// LDE of w columns and the Merkle leaves of its rows (tree level 0; tree.d allocated by
// the caller, one leaf per LDE row); d_keep receives the first keep_cols LDE columns.
// trace is a host pointer when host_trace.
void lde_commit(sg_ctx* c, const uint64_t* trace, bool host_trace, uint64_t w, uint64_t n_trace, uint64_t blowup,
                uint64_t shift, const DevTree& tree, uint64_t* d_keep, uint64_t keep_cols);
// lambdas are host values; n_blocks gates the SHA-256 AIR (the AIR registry uses 1)
void merge_device(sg_ctx* c, int air, const uint64_t* d_lde, uint64_t w, uint64_t n_trace, uint64_t blowup,
                  const uint64_t* lambdas, uint64_t k, int phi_mode, uint64_t* d_c, uint64_t n_blocks = 1);
// Phi + quotient of a hash AIR on a materialised LDE (lambdas: host values).
void merge_hash_device(sg_ctx* c, const HashAir& air, const uint64_t* d_lde, uint64_t n_trace, uint64_t blowup,
                       const uint64_t* lambdas, int phi_mode, uint64_t* d_c, uint64_t n_blocks);
// message -> hash AIR trace -> LDE x blowup (32 in the reference's provers) -> merge ->
// STIR; digest gets air.digest_bytes.
std::vector<uint8_t> prove_hash_message(sg_ctx* c, const HashAir& air, const uint8_t* msg, uint64_t len,
                                        const uint8_t fs_binding[32], int phi_mode, bool self_verify,
                                        uint8_t* digest, uint64_t blowup = 32);
CEval hash_message_ceval(sg_ctx* c, const HashAir& air, const uint8_t* msg, uint64_t len,
                         const uint8_t fs_binding[32], int phi_mode, uint8_t* digest, uint64_t blowup = 32);
// prove_ds_ksk_binding core: message -> SHA-256 AIR trace -> LDE x blowup -> merge -> STIR.
std::vector<uint8_t> prove_sha256_message(sg_ctx* c, const uint8_t* msg, uint64_t len, const uint8_t fs_binding[32],
                                          int phi_mode, bool self_verify, uint8_t digest[32], uint64_t blowup = 32);
std::vector<uint8_t> stir_prove_device(sg_ctx* c, const uint64_t* d_f0, uint64_t n0, const sg_fri_params& p);
// G STIR proofs in lockstep (one launch per stage over all of them): the same n0
// and parameters except the public-input hash, proof g's f0 at d_f0 + g * g_f0;
// proof g's bytes equal stir_prove_device's.
std::vector<std::vector<uint8_t>> stir_prove_group(sg_ctx* c, const uint64_t* d_f0, uint64_t g_f0, uint64_t n0,
                                                   const std::vector<sg_fri_params>& ps);
// RSA-2048 signature-check proof (prove_rsa2048_record_v1.rs for one record,
// stacked_rsa_zone_prover.rs for several): witnesses on the host, trace expanded
// on the device -> LDE x32 -> RSA merge (Phi always evaluated) -> STIR with
// build_params(1024, pi). Inputs: n_records 256-byte big-endian n, s, em each.
std::vector<uint8_t> prove_rsa2048(sg_ctx* c, const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be,
                                   uint64_t n_records, const uint8_t pi[32], bool self_verify, uint64_t blowup = 32);
CEval rsa2048_ceval(sg_ctx* c, const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be, uint64_t n_records,
                    const uint8_t pi[32], uint64_t blowup = 32);
// A power of two in [2, 1024], else SgError.
void check_blowup(uint64_t blowup);
// The host witnesses of n_records records (threads over records).
void rsa_witnesses(const uint8_t* n_be, const uint8_t* s_be, const uint8_t* em_be, uint64_t n_records,
                   std::vector<rsa::RecordW>* recs, std::vector<rsa::RowW>* rows);
// prove_inner_shard / prove_outer_rollup core: HashRollup trace -> LDE x32 -> merge ->
// STIR (stir) or classic DEEP-FRI, with build_params(n0, pi).
std::vector<uint8_t> prove_hash_rollup_host_leaves(sg_ctx* c, const uint64_t* leaves, uint64_t n_leaves,
                                                   const uint8_t pi[32], int phi_mode, bool self_verify,
                                                   bool stir = true);

}  // namespace sg
